// tild_sort.cu — spatial re-ordering of the bead slots of every system of an engine.
//
// The reference keeps beads in file order for its whole run (d_x, device_comm_utils.cu:5-17), so
// every stencil access of its spread and gather lands on an unrelated cache line.  Here the slots
// are re-sorted every `sort_interval` steps by the grid cell of the bead, cells taken in 4x4x4
// bricks (8x8 in 2D) so that a warp's beads share stencil nodes.  The key carries the rank of the
// system's slot range in its high bits and padding slots get the largest cell code, so each
// system keeps its slot range with its beads first.  The sort is stable (CUB radix sort on (key, slot)); every per-bead array
// is permuted and bond partners are renumbered, so the physics never depends on the order: noise
// is keyed by the bead id, and outputs are written by bead id.
#include "tild_internal.cuh"
#include <cub/device/device_radix_sort.cuh>

namespace {

inline unsigned nblk(long long n, int b) { return (unsigned)((n + b - 1) / b); }

// ceil(log2(v)) for v >= 1
__device__ __forceinline__ int ilog2c(int v) { return v <= 1 ? 0 : 32 - __clz(v - 1); }

// Sort key of a slot: the system in the high bits, then the brick of its grid cell, then the cell
// inside the brick (x fastest).  `brick` packs log2 of the brick edges (bits 0-3 x, 4-7 y, 8-11 z,
// each capped by the grid) and bit 12 orders bricks along a Morton curve instead of x-fastest.
__global__ void k_sort_keys(const float4* __restrict__ pos, const int* __restrict__ cta_sys,
                            const SysDev* __restrict__ sysd, int D, int cell_bits, int brick, unsigned* __restrict__ keys,
                            int* __restrict__ vals) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  const int sys = cta_sys[blockIdx.x];
  const Geom& g = sysd[sys].g;
  const float4 p = pos[slot];
  const unsigned pad_code = (1u << cell_bits) - 1u;
  unsigned cell = pad_code;
  if (tild_type_of(p.w) != kPadType) {
    const float xs[3] = {p.x, p.y, p.z};
    int c[3] = {0, 0, 0}, sh[3] = {0, 0, 0}, nb[3] = {1, 1, 1}, bb[3] = {0, 0, 0};
    for (int d = 0; d < D; d++) {
      int v = isfinite(xs[d]) ? (int)(xs[d] / g.dx[d]) : 0;
      c[d] = min(max(v, 0), g.nx[d] - 1);
      sh[d] = min((brick >> (4 * d)) & 15, ilog2c(g.nx[d]));
      nb[d] = (g.nx[d] + (1 << sh[d]) - 1) >> sh[d];
      bb[d] = ilog2c(nb[d]);
    }
    unsigned bidx;
    if (brick >> 12 & 1) {  // Morton order of the bricks: bits interleaved x, y, z
      const int nmax = max(bb[0], max(bb[1], bb[2]));
      bidx = 0;
      int o = 0;
      for (int b = 0; b < nmax; b++)
        for (int d = 0; d < 3; d++)
          if (b < bb[d]) bidx |= (((unsigned)(c[d] >> sh[d]) >> b) & 1u) << o++;
    } else {
      bidx = ((unsigned)(c[2] >> sh[2]) * nb[1] + (unsigned)(c[1] >> sh[1])) * nb[0] + (c[0] >> sh[0]);
    }
    const unsigned local = ((((unsigned)c[2] & ((1u << sh[2]) - 1)) << sh[1]) | ((unsigned)c[1] & ((1u << sh[1]) - 1)))
                               << sh[0] |
                           ((unsigned)c[0] & ((1u << sh[0]) - 1));
    cell = (bidx << (sh[0] + sh[1] + sh[2])) | local;
  }
  keys[slot] = ((unsigned)sysd[sys].slot_rank << cell_bits) | cell;
  vals[slot] = slot;
}

// gather every per-slot array into the new order; new_slot[old] = new
__global__ void k_permute(const int* __restrict__ perm, int n, const float4* __restrict__ p0,
                          const float4* __restrict__ p1, const float* __restrict__ noise, const int* __restrict__ bid,
                          const int* __restrict__ info, const float* __restrict__ q,
                          const curandStateXORWOW_t* __restrict__ xw, float4* __restrict__ p0n, float4* __restrict__ p1n,
                          float* __restrict__ noisen, int* __restrict__ bidn, int* __restrict__ infon,
                          float* __restrict__ qn, curandStateXORWOW_t* __restrict__ xwn, int* __restrict__ new_slot) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
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

__global__ void k_remap_bonds(const int* __restrict__ perm, int n, const int* __restrict__ nbr,
                              const int* __restrict__ info_new, const int* __restrict__ new_slot,
                              const int* __restrict__ bid_new, const int* __restrict__ cta_sys,
                              const SysDev* __restrict__ sysd, int* __restrict__ nbrn, int* __restrict__ slot_of) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int o = perm[s];
  const int nb = info_new[s] & 3;
  for (int k = 0; k < 3; k++) nbrn[3 * (long long)s + k] = (k < nb) ? new_slot[nbr[3 * (long long)o + k]] : 0;
  const int b = bid_new[s];
  if (b >= 0) slot_of[sysd[cta_sys[s / kTile]].bead0 + b] = s;
}

int log2_ceil(long long v) {
  int s = 0;
  while ((1ll << s) < v) s++;
  return s;
}

}  // namespace

int tild_sort_alloc(tild_ctx* c) {
  const size_t n = c->nslots;
  auto A = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes ? bytes : 1) != cudaSuccess; };
  if (A((void**)&c->sort_keys, n * 4) || A((void**)&c->sort_keys_alt, n * 4) || A((void**)&c->sort_vals, n * 4) ||
      A((void**)&c->sort_perm, n * 4) || A((void**)&c->sort_newslot, n * 4) ||
      A((void**)&c->alt_pos[0], n * sizeof(float4)) || A((void**)&c->alt_pos[1], n * sizeof(float4)) ||
      A((void**)&c->alt_noise, n * 12) || A((void**)&c->alt_bead_id, n * 4) || A((void**)&c->alt_info, n * 4) ||
      A((void**)&c->alt_nbr, n * 12) || (c->charge && A((void**)&c->alt_charge, n * 4)) ||
      (c->xorwow && A((void**)&c->alt_xorwow, n * sizeof(curandStateXORWOW_t)))) {
    cudaGetLastError();
    c->err = "device allocation failed: sort buffers";
    return TILD_ERR_OOM;
  }
  // cell code bits: enough for every brick shape the tuner may choose, for the largest system,
  // with the all-ones code left for padding slots
  int cell_bits = 1;
  for (const SysHost& h : c->sys)
    for (int brick : tild_brick_candidates(c->D)) {
      int local = 0, bbits = 0;
      long long nbricks = 1;
      for (int d = 0; d < c->D; d++) {
        const int sh = std::min((brick >> (4 * d)) & 15, log2_ceil(h.g.nx[d]));
        const long long nb = (h.g.nx[d] + (1 << sh) - 1) >> sh;
        local += sh;
        nbricks *= nb;
        bbits += log2_ceil(nb);
      }
      const int bits = local + ((brick >> 12 & 1) ? bbits + 1 : log2_ceil(nbricks + 1));
      cell_bits = std::max(cell_bits, bits);
    }
  const int sys_bits = log2_ceil(c->nsys);
  if (cell_bits + sys_bits > 32) {
    c->err = "spatial sort keys need more than 32 bits (too many systems or too large a grid)";
    return TILD_ERR_UNSUPPORTED;
  }
  c->sort_cell_bits = cell_bits;
  c->sort_bits = std::max(cell_bits + sys_bits, 1);
  size_t tb = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tb, c->sort_keys, c->sort_keys_alt, c->sort_vals, c->sort_perm, c->nslots,
                                  0, c->sort_bits, c->stream);
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

// The permuted arrays become the current ones: every per-slot array trades places with its
// alternate.  A replayed CUDA graph that contains sorts applies the same trades on the host.
void tild_sort_swap_buffers(tild_ctx* c) {
  std::swap(c->pos[0], c->alt_pos[0]);
  std::swap(c->pos[1], c->alt_pos[1]);
  std::swap(c->noise, c->alt_noise);
  std::swap(c->bead_id, c->alt_bead_id);
  std::swap(c->bond_info, c->alt_info);
  std::swap(c->bond_nbr, c->alt_nbr);
  if (c->charge) std::swap(c->charge, c->alt_charge);
  if (c->xorwow) std::swap(c->xorwow, c->alt_xorwow);
}

int tild_sort_beads(tild_ctx* c) {
  if (!c->sort_temp) return TILD_OK;
  const int n = c->nslots;
  const unsigned nb = nblk(n, kTile);
  cudaStream_t st = c->stream;
  k_sort_keys<<<c->n_cta_bead, kTile, 0, st>>>(c->pos[c->cur], c->cta_bead, c->d_sys, c->D, c->sort_cell_bits,
                                               c->sort_brick, c->sort_keys, c->sort_vals);
  c->launches++;
  size_t tb = c->sort_temp_bytes;
  if (cub::DeviceRadixSort::SortPairs(c->sort_temp, tb, c->sort_keys, c->sort_keys_alt, c->sort_vals, c->sort_perm, n,
                                      0, c->sort_bits, st) != cudaSuccess) {
    cudaGetLastError();
    c->err = "radix sort failed";
    return TILD_ERR_CUDA;
  }
  k_permute<<<nb, kTile, 0, st>>>(c->sort_perm, n, c->pos[c->cur], c->pos[c->cur ^ 1], c->noise, c->bead_id,
                                  c->bond_info, c->charge, c->xorwow, c->alt_pos[c->cur], c->alt_pos[c->cur ^ 1],
                                  c->alt_noise, c->alt_bead_id, c->alt_info, c->alt_charge, c->alt_xorwow,
                                  c->sort_newslot);
  k_remap_bonds<<<nb, kTile, 0, st>>>(c->sort_perm, n, c->bond_nbr, c->alt_info, c->sort_newslot, c->alt_bead_id,
                                      c->cta_bead, c->d_sys, c->alt_nbr, c->slot_of);
  c->launches += 2;
  tild_sort_swap_buffers(c);
  c->steps_since_sort = 0;
  c->sorts++;
  return tild_check(c, cudaGetLastError(), "sort") ? TILD_ERR_CUDA : TILD_OK;
}
