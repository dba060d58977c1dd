// Host-side launch wrappers of the device kernels (C++ linkage, internal).
#pragma once
#include <cuda_runtime.h>
#include "sph_internal.cuh"

namespace sph {

// Kernel classes whose persistent grid the autotuner sizes.
enum GridClass { kGridLists = 0, kGridMomentum = 1, kGridContinuity = 2, kGridBoundary = 3, kGridIntegrals = 4,
                 kGridClasses = 5 };

struct DevBatch {
  const SimDev* sims;      // [nsims]
  SimDyn* dyn;             // [nsims]
  const Tile* tiles;       // [ntiles]
  int ntiles;
  int nsims;
  int dim;
  Particles P;
  const FaceDev* faces;
  const SideDev* sides;
  const EdgeDev* edges;    // convex edges of all simulations (3D)
  const double* bit;       // per-sim BoundIntegralTab, 256 x 7 each
  const int* cf_start;     // per global cell: first entry in cf_list
  const int* cf_count;     // per global cell: faces cutting the cell
  const int* cf_list;      // face ids (1-based within the simulation)
  const uint8_t* cell_near;  // per global cell: faces cut the 27-cell block
  int* nlist;              // neighbour lists (see k_neighbour_lists)
  int* ncount;             // entries per particle
  int list_cap4;           // 4-entry chunks reserved per particle (max NMAXPARTJ / 4)
  unsigned long long* counters;  // [0] momentum candidates, [1] momentum pairs,
                                 // [2] continuity candidates, [3] continuity pairs
  int* scan_block_sums;    // scan scratch
  int scan_nblocks;
  int grid_blocks;         // blocks of the persistent particle kernels (default)
  int sms;                 // streaming multiprocessors of the device
  int grid[kGridClasses];  // autotuned blocks per kernel class (0 = grid_blocks)
  int mom_batch;           // momentum pair loop: 1 = several entries' records loaded together, 2 = the same
                           // with two entries' terms on paired FP32 instructions (FP32c; autotuned)
  int con_batch;           // the same for the continuity pair loop (0, 1, 2)
  int c1;                  // some simulation renormalises (C1_BE, 3D): P.BG (and P.BD) allocated
  int c1_divu;             // some simulation renormalises its velocity gradients (C1_divu)
};

enum class KeyKind { Sort = 0, Reference = 1 };

// sorting
void launch_stage(const DevBatch& b, cudaStream_t st);
void launch_bin(const DevBatch& b, KeyKind kind, cudaStream_t st);
void launch_removal(const DevBatch& b, cudaStream_t st);
void launch_scan(const DevBatch& b, int* cell_start, cudaStream_t st);
void launch_sort_reset(const DevBatch& b, cudaStream_t st);
void upload_bit2d(const double* tab, cudaStream_t st);
void launch_place(const DevBatch& b, cudaStream_t st);
void launch_rank_permute(const DevBatch& b, cudaStream_t st);
// the IC of an upload: positions first (destinations kept in P.slot), then the rest
void launch_rank_permute_positions(const DevBatch& b, cudaStream_t st);
void launch_rank_permute_rest(const DevBatch& b, cudaStream_t st);
void launch_rank_reference(const DevBatch& b, const int* cell_start_ref, int* npartord, cudaStream_t st);
// neighbour lists (CalcVarLength replacement)
void launch_neighbour_lists(const DevBatch& b, cudaStream_t st);
void launch_renormalisation(const DevBatch& b, cudaStream_t st);   // C1: fluid part of the matrices
// physics (FP64)
void launch_boundary(const DevBatch& b, cudaStream_t st);
void launch_momentum(const DevBatch& b, bool fused, cudaStream_t st);
void launch_continuity(const DevBatch& b, bool fused, cudaStream_t st);
// physics (FP32-compensated form)
void launch_momentum_f32(const DevBatch& b, bool fused, cudaStream_t st);
void launch_continuity_f32(const DevBatch& b, bool fused, cudaStream_t st);   // pairs + finish
void launch_continuity_f32_pairs(const DevBatch& b, cudaStream_t st);
void launch_continuity_f32_finish(const DevBatch& b, bool fused, cudaStream_t st);
void launch_refresh_f32(const DevBatch& b, cudaStream_t st);
void launch_leapfrog_momentum(const DevBatch& b, cudaStream_t st);
void launch_leapfrog_trajectories(const DevBatch& b, cudaStream_t st);
void launch_leapfrog_continuity(const DevBatch& b, cudaStream_t st);
void launch_eos(const DevBatch& b, cudaStream_t st);
// partial smoothing (TetaV > 1e-9, TetaP > 0): fused = on the step record
// V2/X2 (step graph), else in place (per-call ABI)
void launch_velocity_smoothing(const DevBatch& b, bool fused, bool fp32c, cudaStream_t st);
void launch_pressure_smoothing(const DevBatch& b, bool fp32c, cudaStream_t st);
void launch_dt_reduce(const DevBatch& b, cudaStream_t st);
void launch_finalize(const DevBatch& b, int mode, cudaStream_t st);
void launch_cancel(const DevBatch& b, int sim, cudaStream_t st);
void launch_set_dt(const DevBatch& b, double dt, cudaStream_t st);
void launch_load_laminar(const DevBatch& b, const int* laminar, cudaStream_t st);
void launch_set_clock(const DevBatch& b, double time, int step, double dt, double dt_prev, double dt_average,
                      const int* laminar, cudaStream_t st);
// host <-> device in caller order
void launch_init_from_caller(const DevBatch& b, const double* x, const double* v, const double* rho,
                             const double* p, const double* m, cudaStream_t st);
void launch_init_positions(const DevBatch& b, const double* x, const double* m, cudaStream_t st);
// a fused step's x, v, m from its momentum record (before its sort) to caller order
void launch_scratch_to_caller(const DevBatch& b, double* x, double* v, double* m, cudaStream_t st);
void launch_init_rest(const DevBatch& b, const double* v, const double* rho, const double* p, cudaStream_t st);
void launch_to_caller(const DevBatch& b, double* x, double* v, double* rho, double* p, double* m,
                      double* acc, double* dden, cudaStream_t st);
// verification
void launch_dump_neighbours(const DevBatch& b, int nmaxj, int* counts, int* lists, cudaStream_t st);
void launch_dump_boundary(const DevBatch& b, int max_per, int* ncb, int* clob, double* vals, cudaStream_t st);
void launch_dump_renormalisation(const DevBatch& b, double* bg, double* bd, cudaStream_t st);
void launch_dump_cella(const DevBatch& b, int* cella, cudaStream_t st);
void launch_dump_laminar(const DevBatch& b, int* flags, cudaStream_t st);
// fluid_global_quantities: part [ntiles][8] scratch, out [nsims][8]
void launch_global_quantities(const DevBatch& b, double2* part, double* out, cudaStream_t st);
// FP64 FMA throughput probe: returns flops per launch
double launch_fp64_probe(double* sink, int blocks, cudaStream_t st);
void launch_check_division(unsigned long long n, unsigned long long seed, unsigned long long* bad, double* first,
                           int blocks, cudaStream_t st);
double launch_fp32_probe(float* sink, int blocks, cudaStream_t st);

}  // namespace sph
