/*
 * tild.h — C ABI of the B200-native TILD hot path (libtild.so).
 *
 * The reference program (gpu-tild) has no library boundary: its per-step hot path is a set
 * of argument-less functions acting on process globals.  Each entry point below replaces
 * one of them; the reference interface it stands in for is cited beside it (paths are
 * relative to the gpu-tild source tree).
 *
 *   forces()                  forces.cu:42           -> tild_forces / tild_step
 *   Integrator::Integrate_2() integrator.cu:24-39    -> tild_step
 *   update_pairstyles()       update_pairstyles.cu:3 -> tild_step (ramp is a per-step scalar)
 *   calc_properties()         calc_properties.cu:20  -> tild_observables
 *   Compute::doCompute()      Compute.cu:83          -> tild_sk_accumulate
 *   Compute::writeResults()   Compute.cu:121         -> tild_sk_get
 *   send_3n_to_device()       device_comm_utils.cu:5 -> tild_set_state
 *   cuda_collect_x/rho/f()    device_comm_utils.cu:20-87 -> tild_get_state / tild_get_density / tild_forces
 *   NList::BuildNList()       nlist.cu:99-110        -> tild_nlist_build
 *
 * Conventions
 *  - Every call returns a tild_status; nothing in the library calls exit().  On error the
 *    context keeps a message readable with tild_last_error().
 *  - Host arrays are plain C arrays in the reference's file order: positions are AoS
 *    [ns][dim] float32, bead index = line order of the data file (0-based), types 0-based.
 *  - A context owns all of its device memory and one CUDA stream; it is not thread-safe.
 *  - No torch or CUDA types appear in this header.
 */
#ifndef TILD_H
#define TILD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TILD_ABI_VERSION 1

#define TILD_MAX_TYPES 16
#define TILD_MAX_STYLES 32
#define TILD_MAX_BOND_TYPES 32
#define TILD_MAX_INTEGRATORS 8
#define TILD_MAX_BONDS 3          /* reference MAX_BONDS, globals.h:26 */
#define TILD_MAX_COMPUTES 8

typedef enum {
  TILD_OK = 0,
  TILD_ERR_CUDA = 1,        /* a CUDA / cuFFT call failed (reference: die() after cudaGetLastError) */
  TILD_ERR_NAN = 2,         /* non-finite position or energy (reference: main.cu:189-191 loop break) */
  TILD_ERR_OOM = 3,         /* device allocation failed */
  TILD_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
  TILD_ERR_BAD_INPUT = 5,   /* invalid configuration or argument (reference: die(msg)) */
  TILD_ERR_UNSUPPORTED = 6, /* a configuration the reference accepts but this build rejects */
  TILD_ERR_STATE = 7        /* call made in the wrong order (e.g. step before set_state) */
} tild_status;

/* Pair styles: reference pair_style_*.cu.  Order inside tild_config.styles is free; the
 * reference evaluates Gaussians, Erfs, FieldPhases, GaussianErfs in that order. */
enum {
  TILD_STYLE_GAUSSIAN = 0,      /* pair_style_gaussian.cu:72-90 */
  TILD_STYLE_ERF = 1,           /* pair_style_erf.cu:122-158 */
  TILD_STYLE_GAUSSIAN_ERF = 2,  /* pair_style_gaussian_erf.cu:82-115 */
  TILD_STYLE_FIELDPHASE = 3     /* pair_style_fieldphases.cu:51-185 */
};

enum { TILD_INTEGRATOR_EM = 0, TILD_INTEGRATOR_GJF = 1 };

enum {
  TILD_RNG_PHILOX = 0,  /* counter-based Philox4x32-10 keyed by (seed, bead id): no per-bead state */
  TILD_RNG_XORWOW = 1   /* cuRAND XORWOW states initialised like init_dev_rng (cuda_random_posits.cu:22-30) */
};

enum {
  TILD_TABLES_FP64 = 0,     /* k-space multipliers built in FP64, stored FP32 */
  TILD_TABLES_REF_FP32 = 1  /* multipliers evaluated with the reference's FP32 formulas */
};

/* One non-bonded pair style.  Field meanings follow the input-script lines parsed in
 * read_input.cu:176-416 (types already shifted to 0-based). */
typedef struct {
  int32_t style;           /* TILD_STYLE_* */
  int32_t type1, type2;    /* 0-based particle types */
  int32_t ramp;            /* nonzero: "ramp <final>" given (pair_style.cu:347-367) */
  float prefactor;         /* A (initial_prefactor) */
  float final_prefactor;   /* ramp target */
  float sigma;             /* smearing length as written in the script (the reference squares it) */
  float rp;                /* particle radius R_p (erf, gaussian_erf) */
  int32_t phase, dir, n_periods;  /* fieldphase only */
  int32_t reserved;
} tild_pair_style;

/* One "integrator <group> <name>" line (integrator.cu:24-39).  Groups are "all" or
 * "type k" (group.cu:30-60), so a group is identified by a particle type or -1 for all. */
typedef struct {
  int32_t kind;        /* TILD_INTEGRATOR_* */
  int32_t group_type;  /* -1 = group "all", else 0-based particle type */
} tild_integrator;

typedef struct {
  int32_t dim;                 /* 2 or 3 */
  int32_t nx[3];               /* grid points per dimension (Nx, Ny, Nz) */
  float box[3];                /* box lengths L (box[2] ignored when dim == 2) */
  int32_t ns;                  /* number of beads */
  int32_t ntypes;
  int32_t pmeorder;            /* 0..4; stencil is (pmeorder+1)^dim points */
  float delt;                  /* time step */
  float noise_mag;             /* reference: sqrtf(2*delt) (read_input.cu:93) */
  uint64_t seed;               /* rand_seed */
  int32_t rng;                 /* TILD_RNG_* */
  int32_t max_steps;           /* only used by prefactor ramps */
  int32_t n_styles;
  tild_pair_style styles[TILD_MAX_STYLES];
  int32_t do_charges;          /* "charges <bjerrum> <smearing>" given */
  float bjerrum;
  float smearing;
  int32_t n_bond_types;
  float bond_k[TILD_MAX_BOND_TYPES];
  float bond_req[TILD_MAX_BOND_TYPES];
  float mass[TILD_MAX_TYPES];
  float diff[TILD_MAX_TYPES];  /* diffusivity, default 1 */
  int32_t n_integrators;
  tild_integrator integrators[TILD_MAX_INTEGRATORS];
  int32_t table_mode;          /* TILD_TABLES_* */
  int32_t sort_interval;       /* steps between spatial re-sorts of the beads; 0 = default, <0 = never */
  int32_t flags;               /* reserved, set 0 */
  int32_t reserved[7];
} tild_config;

/* Observables of calc_properties() (calc_properties.cu:20-116), reduced in FP64.
 * Non-bonded terms use the densities of the last force evaluation, bond terms the current
 * positions, exactly as the reference does at log_freq. */
typedef struct {
  double upe;                          /* total: sum of style energies + electrostatic + bond */
  double ubond;                        /* bonds.cu:3-52 */
  double uelec;                        /* calc_properties.cu:106-116 (0 without charges) */
  double ptens[6];                     /* 3D: xx yy zz xy xz yz; 2D: xx yy xy */
  double bond_vir[6];
  double style_energy[TILD_MAX_STYLES];   /* PairStyle::CalcEnergy, pair_style.cu:204-233 */
  double style_virial[TILD_MAX_STYLES][6];/* PairStyle::CalcVirial, pair_style.cu:235-260 */
  int64_t step;
  int32_t n_styles;
  int32_t n_p_comps;
} tild_obs;

typedef struct tild_ctx tild_ctx;

/* ---- library ---------------------------------------------------------------------- */
int32_t tild_abi_version(void);
const char* tild_status_string(int32_t status);
const char* tild_last_error(const tild_ctx* ctx);

/* ---- setup: replaces initialize() (initialize.cu:20-85) ---------------------------- */
/* Validates cfg, allocates device state on `device`, builds k-space tables in FP64. */
int32_t tild_create(const tild_config* cfg, int32_t device, tild_ctx** out);
int32_t tild_destroy(tild_ctx* ctx);

/* Topology: replaces send_box_params_to_device() (device_comm_utils.cu:90-140).
 * types[ns]; charges[ns] (NULL unless do_charges); n_bonds[ns];
 * bonded_to[ns*3], bond_type[ns*3] in the layout built by read_config
 * (config_utils.cu:111-123: both directions of every bond stored). */
int32_t tild_set_topology(tild_ctx* ctx, const int32_t* types, const float* charges,
                          const int32_t* n_bonds, const int32_t* bonded_to,
                          const int32_t* bond_type);

/* Positions [ns][dim].  xo and prev_noise may be NULL: then xo = x and prev_noise = 0,
 * which is what send_3n_to_device() + allocate_device_memory() do. */
int32_t tild_set_state(tild_ctx* ctx, const float* x, const float* xo, const float* prev_noise);
int32_t tild_get_state(tild_ctx* ctx, float* x, float* xo, float* prev_noise);

/* ---- per step ------------------------------------------------------------------------ */
/* forces(): spread, convolve, gather, bonds, for the current positions.  Writes per-bead
 * forces [ns][dim] to f (host) if f != NULL.  Beads do not move. */
int32_t tild_forces(tild_ctx* ctx, float* f);

/* nsteps x { forces(); Integrate_2() for every integrator; update_pairstyles(); } with the
 * step counter advancing by one each time (main.cu:106-201 minus I/O). */
int32_t tild_step(tild_ctx* ctx, int32_t nsteps);

/* Current step counter (0 after create). */
int32_t tild_get_step(tild_ctx* ctx, int64_t* step);
int32_t tild_set_step(tild_ctx* ctx, int64_t step);

/* calc_properties(). */
int32_t tild_observables(tild_ctx* ctx, tild_obs* out);

/* Density grids of the last force evaluation: rho[ntypes][M] (+ charge grid [M] appended
 * when do_charges).  M = prod(nx), x fastest. */
int32_t tild_get_density(tild_ctx* ctx, float* rho);

/* Assignment stencil of every bead for the current positions, in the order d_charge_grid
 * stores them (device_grid_utils.cu:232-343): inds[ns*S], w[ns*S] (w = product of weights
 * / gvol).  Either pointer may be NULL. */
int32_t tild_get_stencil(tild_ctx* ctx, int32_t* inds, float* w);

/* ---- computes: avg_sk (Compute.cu:83-138) --------------------------------------------- */
/* Accumulates rho_k * rho_k / M (the reference's product, not |rho_k|^2) of `type` from the
 * densities of the last force evaluation into accumulator `slot` (0..TILD_MAX_COMPUTES-1). */
int32_t tild_sk_accumulate(tild_ctx* ctx, int32_t slot, int32_t type);
/* Full-spectrum average accumulated/ncalls as interleaved complex [M][2] (FP64); ncalls out. */
int32_t tild_sk_get(tild_ctx* ctx, int32_t slot, double* sk, int32_t* ncalls);

/* ---- neighbour list (nlist.cu) ---------------------------------------------------------- */
/* Builds the cell list and neighbour list of the beads of group `group_type` (-1 = all)
 * with cutoff rc, as NList::Initialize/BuildNList define them (nlist.cu:64-161).
 * Outputs (host): cell_of[ns] (-1 for beads outside the group), neigh_count[ns],
 * neigh[ns*cell_max] (neighbour bead ids, each row sorted ascending — the reference's row
 * order is atomic-order dependent).  cell_max_out receives CELL_MAX.  Any output may be
 * NULL; call once with neigh == NULL to learn cell_max. */
int32_t tild_nlist_build(tild_ctx* ctx, float rc, int32_t group_type, int32_t* cell_of,
                         int32_t* neigh_count, int32_t* neigh, int32_t* cell_max_out);

/* ---- measurement ------------------------------------------------------------------------- */
/* Runs nsteps steps exactly as tild_step does, recording a CUDA event pair around every
 * stage on the context's stream.  stage_ms[i] = total milliseconds of stage i;
 * stage_names receives a comma-separated list of stage names (buffer of name_cap bytes). */
int32_t tild_profile_steps(tild_ctx* ctx, int32_t nsteps, double* stage_ms, int32_t max_stages,
                           int32_t* n_stages, char* stage_names, int32_t name_cap);
/* Runs nsteps steps as one timed region (events on the context stream), returns ms. */
int32_t tild_time_steps(tild_ctx* ctx, int32_t nsteps, double* ms);
/* Number of kernels this library launched since create (cuFFT's internal kernels excluded). */
int32_t tild_kernel_launches(tild_ctx* ctx, int64_t* count);
/* Blocks until the context stream is idle; reports any device-side status flag. */
int32_t tild_sync(tild_ctx* ctx);

/* ---- batches: many independent systems advanced together ------------------------------------ */
/* No single reference call corresponds: the reference runs one system per process.  A batch
 * advances every system with one launch per stage (spread, k-space multiply, gather) and one
 * batched cuFFT plan per grid shape.  Systems must share dim, pmeorder and rng; everything else
 * (box, grid, types, styles, bonds, integrators, seed, time step) is per system.  Per-system
 * calls take the system index `sys` (0..nsys-1) and mirror the single-system calls above. */
typedef struct tild_batch tild_batch;
int32_t tild_batch_create(const tild_config* cfgs, int32_t nsys, int32_t device, tild_batch** out);
int32_t tild_batch_destroy(tild_batch* b);
const char* tild_batch_last_error(const tild_batch* b);
int32_t tild_batch_set_topology(tild_batch* b, int32_t sys, const int32_t* types, const float* charges,
                                const int32_t* n_bonds, const int32_t* bonded_to, const int32_t* bond_type);
int32_t tild_batch_set_state(tild_batch* b, int32_t sys, const float* x, const float* xo, const float* prev_noise);
int32_t tild_batch_get_state(tild_batch* b, int32_t sys, float* x, float* xo, float* prev_noise);
/* Systems marked inactive keep their state and are skipped by every per-step kernel. */
int32_t tild_batch_set_active(tild_batch* b, int32_t sys, int32_t active);
int32_t tild_batch_set_step(tild_batch* b, int32_t sys, int64_t step);
int32_t tild_batch_get_step(tild_batch* b, int32_t sys, int64_t* step);
/* nsteps steps of every active system. */
int32_t tild_batch_step(tild_batch* b, int32_t nsteps);
/* One force evaluation of every active system; forces of system `sys` to f if f != NULL. */
int32_t tild_batch_forces(tild_batch* b, int32_t sys, float* f);
int32_t tild_batch_observables(tild_batch* b, int32_t sys, tild_obs* out);
int32_t tild_batch_get_density(tild_batch* b, int32_t sys, float* rho);
int32_t tild_batch_time_steps(tild_batch* b, int32_t nsteps, double* ms);
int32_t tild_batch_sync(tild_batch* b);
/* avg_sk of one system (tild_sk_accumulate / tild_sk_get for system `sys`). */
int32_t tild_batch_sk_accumulate(tild_batch* b, int32_t sys, int32_t slot, int32_t type);
int32_t tild_batch_sk_get(tild_batch* b, int32_t sys, int32_t slot, double* sk, int32_t* ncalls);

/* ---- slots: continuous batching (no reference counterpart) ----------------------------------- */
/* A slot batch reserves capacity[s] >= cfgs[s].ns beads for system s, so that tild_batch_load can
 * later put another system of the same grid shape into slot s while the others keep running. */
int32_t tild_batch_create_slots(const tild_config* cfgs, const int32_t* capacity, int32_t nsys, int32_t device,
                                tild_batch** out);
int32_t tild_batch_capacity(tild_batch* b, int32_t sys, int32_t* capacity);
/* Replaces the system of slot `sys` by cfg.  cfg must share the slot's dim, pmeorder, rng, grid
 * nx, ntypes and do_charges, and its number of FFT pair styles and of fieldphase styles, with
 * cfg->ns <= the slot's capacity; box, style parameters, bonds, masses, integrators, seed, time
 * step and max_steps may differ.  The slot's k-space tables are rebuilt (nothing is allocated),
 * its avg_sk accumulators are cleared, its step counter is 0 and it is left inactive without
 * topology or state: tild_batch_set_topology, tild_batch_set_state and tild_batch_set_active
 * follow.  Waits for the batch's stream. */
int32_t tild_batch_load(tild_batch* b, int32_t sys, const tild_config* cfg);
/* System `sys` leaves the active set on the device when its step counter reaches stop_at
 * (-1: never), so a stepping call may run past a system's last step: that system takes exactly
 * stop_at - step steps.  Step counters and activity are read back after every stepping call. */
int32_t tild_batch_set_stop(tild_batch* b, int32_t sys, int64_t stop_at);
int32_t tild_batch_get_active(tild_batch* b, int32_t sys, int32_t* active);

/* ---- schedule tuning (no reference counterpart) --------------------------------------------- */
/* Settings that change how, not what, the step computes: densities are fixed-point sums and
 * every other kernel is per bead or per grid point, so results are bitwise the same under any of
 * them. */
enum { TILD_SPREAD_TILED = 0, TILD_SPREAD_DIRECT = 1 };
enum { TILD_GATHER_DIRECT = 0, TILD_GATHER_BOX = 1 };
enum { TILD_FIELD_LINEAR = 0, TILD_FIELD_BRICK = 1 };
typedef struct tild_tune {
  int32_t spread_mode;    /* order >= 2: shared-memory box per 256 beads (TILED) or 64-bit global atomics (DIRECT) */
  int32_t spread_cap;     /* shared box of the tiled spread, 32-bit words, 1024..12288, a multiple of 4 */
  int32_t sort_interval;  /* steps between spatial sorts; 0 = never (only when the context sorts) */
  int32_t fft_streams;    /* auxiliary streams the per-grid-shape FFTs are spread over (0..8) */
  int32_t gather_mode;    /* order >= 2: stencil nodes read from global memory (DIRECT) or from a shared
                             box each CTA stages first (BOX) */
  int32_t gather_cap;     /* shared box of the box gather, float4 nodes, 1024..3072 */
  int32_t sort_brick;     /* sort key bricks: log2 edges x | y<<4 | z<<8, bit 12 = Morton order of the
                             bricks; 3D 0x222 (default), 0x1222, 0x1113, 0x1123; 2D 0x033 (default),
                             0x1033, 0x1014 */
  int32_t field_layout;   /* node order of the force field the gather reads: x-fastest (LINEAR) or 4x4x4
                             bricks of consecutive nodes (BRICK, 3D; the box gather needs LINEAR) */
  int32_t fft_pipeline;   /* several grid shapes: 0 runs each stage for all shapes before the next;
                             1 runs each shape's fixed-point conversion, R2C, k-space multiply, C2R
                             and interleave in sequence on its own stream; 2 runs each shape's whole
                             step (spread to gather) on its stream (without fieldphase styles) */
  int32_t spread_ahead;   /* 1: an integrating step's gather (DIRECT) also spreads the updated positions
                             for the next step, which then runs no spread kernel; 0: a spread kernel
                             at the start of every step */
  double ms_per_step;     /* tild_autotune: measured step time with these settings */
} tild_tune;
int32_t tild_get_tune(tild_ctx* ctx, tild_tune* out);
int32_t tild_set_tune(tild_ctx* ctx, const tild_tune* t);
/* Times candidate settings (coordinate descent over spread mode and box, gather mode and box, force
 * field layout, sort bricks, sort interval and FFT streams, each trial trial_steps steps after one graph period of warm-up) and keeps the fastest.
 * The state of every system (positions, x_{n-1}, noise, step counters, activity) is restored
 * afterwards, so tuning does not advance the simulation.  Not available with TILD_RNG_XORWOW (the
 * generator states would advance). */
int32_t tild_autotune(tild_ctx* ctx, int32_t trial_steps, tild_tune* best);
int32_t tild_batch_autotune(tild_batch* b, int32_t trial_steps, tild_tune* best);
int32_t tild_batch_get_tune(tild_batch* b, tild_tune* out);
int32_t tild_batch_set_tune(tild_batch* b, const tild_tune* t);

/* ---- asynchronous snapshots for output writers ----------------------------------------------- */
/* The reference copies positions and densities to the host and formats its output files between
 * steps with the device idle (cuda_collect_x / cuda_collect_rho, device_comm_utils.cu:20-37;
 * write_lammps_traj, config_utils.cu:366-403; write_binary, io_utils.cu:85-134).  Here a snapshot
 * captures the current positions x[ns][Dim] (bead order) and/or the densities rho[(T+C)][M] of the
 * last force evaluation into a device buffer in stream order, and a separate copy stream moves
 * them to the host arrays while the context keeps stepping.  x or rho may be NULL.  Host arrays
 * should be page-locked (tild_host_alloc) for the copy to overlap with stepping.  *ticket names
 * the snapshot; tild_snapshot_wait(ctx, ticket) blocks until it is in the host arrays and may be
 * called from a writer thread other than the one driving the context.  At most
 * TILD_SNAPSHOT_SLOTS snapshots are in flight: a further call first waits for the oldest. */
#define TILD_SNAPSHOT_SLOTS 4
int32_t tild_snapshot_async(tild_ctx* ctx, float* x, float* rho, int64_t* ticket);
int32_t tild_snapshot_wait(tild_ctx* ctx, int64_t ticket);
int32_t tild_batch_snapshot_async(tild_batch* b, int32_t sys, float* x, float* rho, int64_t* ticket);
int32_t tild_batch_snapshot_wait(tild_batch* b, int64_t ticket);
/* Page-locked host memory (cudaMallocHost / cudaFreeHost); NULL when it cannot be had. */
void* tild_host_alloc(size_t bytes);
void tild_host_free(void* p);

/* ---- allocation-free entry point ----------------------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device memory (code that
 * runs inside another framework's allocator, or after device allocation has been closed): the
 * bond energy and bond virial that host_bonds computes, from positions and topology the caller
 * already holds on the device, with no cudaMalloc, cudaFree or allocating library call.  Its
 * scratch is a fixed device array of TILD_NOALLOC_MAX_BLOCKS x 7 doubles (229 KB) that every GPU
 * loading the library keeps until exit, so ns is limited to TILD_NOALLOC_MAX_BEADS; larger ns
 * returns TILD_ERR_BAD_INPUT.  All calls share that array: calls that overlap on the GPU race.
 * Every call made outside stream capture looks the array's device address up again (so a device
 * reset between calls is harmless); a call on a capturing stream reuses the address the last
 * uncaptured call on that device and context found, and returns TILD_ERR_STATE if there was
 * none: make one call outside capture first, and again after a device reset.  A CUDA error
 * already pending on the calling thread is left pending and reported as TILD_ERR_CUDA with
 * nothing launched.  Corrupt topology (a bond count outside 0..3, a partner or bond type out of
 * range) makes d_out[0] NaN.
 *   d_x[ns*dim] float, d_n_bonds[ns], d_bonded_to[ns*3], d_bond_type[ns*3]: device arrays in the
 *   read_config layout; box[3], bond_k[], bond_req[]: host arrays; d_out (device, FP64):
 *   d_out[0] = bond energy, d_out[1..nP] = bond virial / (V * dim) (nP = 6 in 3D, 3 in 2D);
 *   stream: a cudaStream_t or NULL.  The call is stream-ordered and does not synchronise. */
#define TILD_NOALLOC_MAX_BLOCKS 4096
#define TILD_NOALLOC_MAX_BEADS (TILD_NOALLOC_MAX_BLOCKS * 256)
int32_t tild_bond_observables_noalloc(const float* d_x, const int32_t* d_n_bonds, const int32_t* d_bonded_to,
                                      const int32_t* d_bond_type, int32_t ns, int32_t dim, const float* box,
                                      int32_t n_bond_types, const float* bond_k, const float* bond_req,
                                      double* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TILD_H */
