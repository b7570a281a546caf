// tild_sort.cu — spatial re-ordering of the bead slots.
//
// The reference keeps beads in file order for its whole run (d_x, device_comm_utils.cu:5-17), so
// every stencil access of its spread and gather lands on an unrelated cache line.  Here the slots
// are re-sorted every `sort_interval` steps by the grid cell of the bead, cells taken in 4x4x4
// bricks (8x8 in 2D) so that a warp's beads share stencil points.  The sort is stable (CUB radix
// sort on (key, slot)), every per-bead array is permuted and bond partners are renumbered, so the
// physics never depends on the order: noise is keyed by the original bead id, and outputs are
// written by bead id.
#include "tild_internal.cuh"
#include <cub/device/device_radix_sort.cuh>

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

struct KeyGeom {
  int nb[3];     // bricks per axis
  int shift[3];  // log2 of the brick edge
  int D;
};

__global__ void k_sort_keys(const float4* __restrict__ pos, int ns, Geom g, KeyGeom kg, unsigned* __restrict__ keys,
                            int* __restrict__ vals) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const float4 p = pos[s];
  const float xs[3] = {p.x, p.y, p.z};
  int c[3] = {0, 0, 0};
  for (int d = 0; d < kg.D; d++) {
    int v = isfinite(xs[d]) ? (int)(xs[d] / g.dx[d]) : 0;
    v = min(max(v, 0), g.nx[d] - 1);
    c[d] = v;
  }
  unsigned key;
  if (kg.D == 3) {
    const unsigned bx = c[0] >> kg.shift[0], by = c[1] >> kg.shift[1], bz = c[2] >> kg.shift[2];
    const unsigned lx = c[0] & ((1 << kg.shift[0]) - 1), ly = c[1] & ((1 << kg.shift[1]) - 1),
                   lz = c[2] & ((1 << kg.shift[2]) - 1);
    const unsigned brick = (bz * kg.nb[1] + by) * kg.nb[0] + bx;
    key = (brick << (kg.shift[0] + kg.shift[1] + kg.shift[2])) |
          (((lz << kg.shift[1]) | ly) << kg.shift[0]) | lx;
  } else {
    const unsigned bx = c[0] >> kg.shift[0], by = c[1] >> kg.shift[1];
    const unsigned lx = c[0] & ((1 << kg.shift[0]) - 1), ly = c[1] & ((1 << kg.shift[1]) - 1);
    const unsigned brick = by * kg.nb[0] + bx;
    key = (brick << (kg.shift[0] + kg.shift[1])) | (ly << kg.shift[0]) | lx;
  }
  keys[s] = key;
  vals[s] = s;
}

// gather every per-bead array into the new order; new_slot[old] = new
__global__ void k_permute(const int* __restrict__ perm, int ns, const float4* __restrict__ p0,
                          const float4* __restrict__ p1, const float* __restrict__ noise, const int* __restrict__ bid,
                          const int* __restrict__ info, const float* __restrict__ q,
                          const curandStateXORWOW_t* __restrict__ xw, float4* __restrict__ p0n, float4* __restrict__ p1n,
                          float* __restrict__ noisen, int* __restrict__ bidn, int* __restrict__ infon,
                          float* __restrict__ qn, curandStateXORWOW_t* __restrict__ xwn, int* __restrict__ new_slot) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int o = perm[s];
  p0n[s] = p0[o];
  p1n[s] = p1[o];
  noisen[3 * (long long)s] = noise[3 * (long long)o];
  noisen[3 * (long long)s + 1] = noise[3 * (long long)o + 1];
  noisen[3 * (long long)s + 2] = noise[3 * (long long)o + 2];
  bidn[s] = bid[o];
  infon[s] = info[o];
  if (q) qn[s] = q[o];
  if (xw) xwn[s] = xw[o];
  new_slot[o] = s;
}

__global__ void k_remap_bonds(const int* __restrict__ perm, int ns, const int* __restrict__ nbr,
                              const int* __restrict__ info_new, const int* __restrict__ new_slot,
                              const int* __restrict__ bid_new, int* __restrict__ nbrn, int* __restrict__ slot_of) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int o = perm[s];
  const int nb = info_new[s] & 3;
  for (int k = 0; k < 3; k++) nbrn[3 * (long long)s + k] = (k < nb) ? new_slot[nbr[3 * (long long)o + k]] : 0;
  slot_of[bid_new[s]] = s;
}

int log2_ceil(int v) {
  int s = 0;
  while ((1 << s) < v) s++;
  return s;
}

}  // namespace

int tild_sort_alloc(tild_ctx* c) {
  const size_t ns = c->ns;
  auto A = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes ? bytes : 1) != cudaSuccess; };
  if (A((void**)&c->sort_keys, ns * 4) || A((void**)&c->sort_keys_alt, ns * 4) || A((void**)&c->sort_vals, ns * 4) ||
      A((void**)&c->sort_perm, ns * 4) || A((void**)&c->sort_newslot, ns * 4) ||
      A((void**)&c->alt_pos[0], ns * sizeof(float4)) || A((void**)&c->alt_pos[1], ns * sizeof(float4)) ||
      A((void**)&c->alt_noise, ns * 12) || A((void**)&c->alt_bead_id, ns * 4) || A((void**)&c->alt_info, ns * 4) ||
      A((void**)&c->alt_nbr, ns * 12) || (c->C && A((void**)&c->alt_charge, ns * 4)) ||
      (c->xorwow && A((void**)&c->alt_xorwow, ns * sizeof(curandStateXORWOW_t)))) {
    cudaGetLastError();
    c->err = "device allocation failed: sort buffers";
    return TILD_ERR_OOM;
  }
  // brick edges: 4 cells in 3D, 8 in 2D, never larger than the grid
  KeyGeom kg;
  kg.D = c->D;
  int bits = 0;
  for (int d = 0; d < 3; d++) {
    const int edge = (d < c->D) ? std::min(c->D == 3 ? 4 : 8, 1 << log2_ceil(c->g.nx[d])) : 1;
    kg.shift[d] = log2_ceil(edge);
    kg.nb[d] = (c->g.nx[d] + edge - 1) / edge;
  }
  bits = log2_ceil(kg.nb[0] * kg.nb[1] * kg.nb[2]) + kg.shift[0] + kg.shift[1] + kg.shift[2];
  c->sort_bits = std::max(bits, 1);
  memcpy(c->sort_kg, &kg, sizeof(kg));
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, c->sort_keys, c->sort_keys_alt, c->sort_vals, c->sort_perm, c->ns, 0,
                                  c->sort_bits, c->stream);
  if (cudaMalloc(&c->sort_temp, tb ? tb : 1) != cudaSuccess) {
    cudaGetLastError();
    c->err = "device allocation failed: sort scratch";
    return TILD_ERR_OOM;
  }
  c->sort_temp_bytes = tb;
  return TILD_OK;
}

void tild_sort_free(tild_ctx* c) {
  void* ptrs[] = {c->sort_keys, c->sort_keys_alt, c->sort_vals, c->sort_perm, c->sort_newslot, c->alt_pos[0],
                  c->alt_pos[1], c->alt_noise, c->alt_bead_id, c->alt_info, c->alt_nbr, c->alt_charge, c->alt_xorwow,
                  c->sort_temp};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

int tild_sort_beads(tild_ctx* c) {
  if (!c->sort_temp) return TILD_OK;
  KeyGeom kg;
  memcpy(&kg, c->sort_kg, sizeof(kg));
  const unsigned nb = nblk(c->ns, 256);
  cudaStream_t st = c->stream;
  k_sort_keys<<<nb, 256, 0, st>>>(c->pos[c->cur], c->ns, c->g, kg, c->sort_keys, c->sort_vals);
  c->launches++;
  size_t tb = c->sort_temp_bytes;
  if (cub::DeviceRadixSort::SortPairs(c->sort_temp, tb, c->sort_keys, c->sort_keys_alt, c->sort_vals, c->sort_perm,
                                      c->ns, 0, c->sort_bits, st) != cudaSuccess) {
    cudaGetLastError();
    c->err = "radix sort failed";
    return TILD_ERR_CUDA;
  }
  k_permute<<<nb, 256, 0, st>>>(c->sort_perm, c->ns, c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id,
                                c->bond_info, c->charge, c->xorwow, c->alt_pos[c->cur], c->alt_pos[c->cur ^ 1],
                                c->alt_noise, c->alt_bead_id, c->alt_info, c->alt_charge, c->alt_xorwow,
                                c->sort_newslot);
  k_remap_bonds<<<nb, 256, 0, st>>>(c->sort_perm, c->ns, c->bond_nbr, c->alt_info, c->sort_newslot, c->alt_bead_id,
                                    c->alt_nbr, c->slot_of);
  c->launches += 2;
  std::swap(c->pos[0], c->alt_pos[0]);
  std::swap(c->pos[1], c->alt_pos[1]);
  std::swap(c->noise, c->alt_noise);
  std::swap(c->bead_id, c->alt_bead_id);
  std::swap(c->bond_info, c->alt_info);
  std::swap(c->bond_nbr, c->alt_nbr);
  if (c->C) std::swap(c->charge, c->alt_charge);
  if (c->xorwow) std::swap(c->xorwow, c->alt_xorwow);
  c->last_sort_step = c->step;
  c->sorts++;
  return tild_check(c, cudaGetLastError(), "sort") ? TILD_ERR_CUDA : TILD_OK;
}
