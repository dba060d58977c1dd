// Internal device-side definitions shared by the CUDA translation units.
//
// Design (B200, sm_100a):
//  * Particles live on the device in cell-sorted structure-of-arrays order.
//    The sort key of a cell (i,j,k) (1-based, CellNumber.f90 numbering) is
//      key = ((j-1)*ni + (i-1))*nk + (k-1)         (z fastest, then x, then y)
//    so that for a fixed (y,x) neighbour column the three cells k-1..k+1 are
//    one contiguous run.  Visiting the 9 (3D) or 3 (2D) runs in (y, x) order
//    and each run front to back reproduces exactly the neighbour order of
//    CalcVarLength.f90:173-269 (jrang -> irang -> krang, then NPartOrd order,
//    which is increasing particle index inside a cell); inside a cell the
//    sort orders particles by their caller index, like OrdGrid1's stable
//    scatter.  The FP64 pair sums therefore run in the reference's order.
//  * No neighbour lists are materialised: every pair pass recomputes the
//    distance test and kernel values (the reference stores 60 B per pair
//    slot, CalcVarLength.f90 / Gest_Trans.f90:138-166).
//  * Several independent simulations can share one launch: every array is
//    the concatenation of the simulations' segments and a block only ever
//    works on one simulation (tile table), reading its SimDev into shared
//    memory.  A single simulation is the one-entry case.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sph {

constexpr int kBlock = 256;          // threads per block of the particle kernels
constexpr int kMaxFaceNodes = 4;
constexpr int kBitRows = 256;        // BITrows = FI_STEPS * TETA_STEPS
constexpr int kKtRows = 40;          // INT_KERNELTABLE
constexpr int kMaxCloseSides = 4;    // MAXCLOSEBOUNDSIDES
constexpr int kMaxLocalFaces = 16;   // per-thread close-face buffer (3D)

// Per-simulation constants (read-only during a step).
struct SimDev {
  double extr_lo[3];      // Grid%extr(:,1)
  double dcd[3];          // Grid%dcd
  int ncd[3];             // Grid%ncd
  int dim;
  int cell_off;           // first global cell of this simulation
  int ncells;             // Grid%nmax; the cell ncells is the removal bin
  int p_off;              // first particle slot
  int cap;                // particle slots reserved
  int nmaxpartj;          // NMAXPARTJ
  int maxcb;              // MAXCLOSEBOUNDFACES (3D) / MAXCLOSEBOUNDSIDES (2D)
  int bdt_quota;          // BoundaryDataTab entries this simulation may take from the pool
  int ioff;               // slab of a decomposed simulation: local x cell i is global cell i + ioff
                          // (extr_lo and dcd stay the whole grid's, so cells are assigned as in it)
  int face_off, nfaces;   // faces (3D)
  int side_off, nsides;   // sides (2D)
  int edge_off, nedges;   // convex edges (3D)
  int dt_alfa_mon, density_thresholds;
  double h, doubleh, squareh, square_doubleh, eta, eta2;
  double coefke, coefkacl, ke_coef, kacl_coef;
  double dx, den0, eps, k_over_rho0, celerita, alfa_mon, kin_visc, p_ref;
  double grav[3];
  double cfl, vsc_coeff, pesodt;
  double forcing_aw2;     // A (2 pi / T)^2 of the lateral tank forcing (0: none)
  double forcing_w;       // 2 pi / T
  double teta_p, teta_v;  // input_any_t%TetaP, TetaV (partial smoothing)
  int c1_be, c1_divu;     // input_any_t%C1_BE, %C1_divu (renormalisation, 3D)
  double invb_det_thresh; // input_any_t%invB_det_thresh
  double c1_w1a, c1_w1b, c1_w2;  // grad_W_sub.f90 factors 1/(pi h^3), 3/(4 pi h^3), 15/(64 pi h^3)
  double zpmin;           // 0.05 h, ComputeBoundaryVolumeIntegrals_P0.f90
  double ktdelta;         // kernel-table step
  double rcp_h, rcp_squareh, rcp_ktdelta;  // RN(1/h), RN(1/h^2), RN(1/ktdelta): divisors of div_rn
  double rcp_dcd[3];      // RN(1/dcd): particle_cell's divisions
  float dcdf[3];          // (float)dcd: cell origins differ by multiples of it
  float rr_lo, rr_hi;     // FP32 screening band around (2h)^2 (see sph_api.cu)
  int narrow_z;           // z cells narrower than 2h: a candidate two cells away can lie within 2h
  int ring_skip;          // boundary quadrature: a ring's later points skip the refresh test (see face_integrals)
  double kerneltab[kKtRows + 1][5];
};

// Per-simulation mutable scalars.
struct SimDyn {
  double dt, dt_prev, dtvel, dt_average, time;
  unsigned long long dtmin_bits;   // atomicMin of positive doubles
  int nag;                         // particles in the grid
  int step;                        // on_going_time_step (completed steps)
  int n_out;                       // out-of-grid particles found this pass
  int removed_total;               // EpOrdGrid
  int warnings;
  int status;
  int ncbf_max;
  int max_neigh;
  int bdt_used;
  int bdt_sim_used;                // entries this simulation took in the current pass
  int pad_used;
  int frozen;                      // reached t_end, failed or cancelled: state kept, no longer advanced
  double t_end;                    // 0 = run without end
  double geff[3];                  // body force of the next step: grav (+ tank forcing)
};

// Solid face (TyBoundaryFace) prepared on the host.
struct FaceDev {
  double T[3][3];         // T[row][col]; column 3 is the inward normal
  double GXref[3];        // Node(nodes)%GX, the local origin
  double AA[2], BB[2], CC[2];  // LocalNormalCoordinates.f90 line coefficients
  double usu_due_area;    // 1 / ((3-fkod) * Area)
  double velocity[3];
  double slip;            // BC_shear_stress_input
  int fkod;               // nodes - 2
  int laminar_no_slip_check;
  int zone_type;
  int pad;
};

// Convex edge shared by two solid faces (TyBoundaryConvexEdge), found on the
// host as FindBoundaryConvexEdges3D.f90 does.
struct EdgeDev {
  int face[2];            // the two faces, 1-based within the simulation
  double gx[3];           // node(1)%GX
  double comp[3];         // node(2)%GX - node(1)%GX
  double length;
};

// Boundary side (TyBoundarySide, 2D) prepared on the host.
struct SideDev {
  double v1[2];           // vertex 1 (x, z)
  double sss[2], nnn[2];  // T(acix,1), T(acix,3)
  double length;
  double RN[2][2];        // RN(acix,acix)
  double velocity[3];
  double angle;
  double slip;
  int previous_side;      // 1-based within the simulation, 0 = none
  int laminar_no_slip_check;
  int zone_type;
  int pad;
};

// One BoundaryDataTab entry (TyBoundaryData).
struct BdtEntry {
  double loc[3];          // LocXYZ
  double bi[8];           // BoundaryIntegral(1:8)
  double ig[9];           // IntGiWrRdV, row-major [r][c]
  int clobonum;           // face / side index within the simulation, 1-based
  int pad;
};

// Work tile: a block processes particles [start, start+count) of sim.
struct Tile {
  int sim;
  int start;
  int count;
  int pad;
};

// Device view of the particle storage.
struct Particles {
  double4* X;       // x, y, z, mass          (sorted)
  float4* XF;       // offset from the cell origin in FP32, w = the cell's k index (as a float)
  float4* VF;       // FP32 form: vx, vy, vz, m/rho
  float4* RF;       // FP32 form: rho, p/rho^2, m, 0
  float2* RM;       // FP32c momentum record: rho, p/rho^2 (m_j = rho_j * VF.w, VF.w kept current)
  double4* V;       // vx, vy, vz, rho (density entering the continuity pass)
  double2* RP;      // current rho, p
  int* I;           // caller index (1-based)
  uint8_t* L;       // laminar_flag
  // scratch record written by the momentum pass, permuted back by the sort
  double4* X2;
  double4* V2;
  double* P2;
  int* I2;
  uint8_t* L2;
  // boundary table
  int* bdt_count;   // per particle
  int* bdt_start;
  BdtEntry* bdt;
  int bdt_cap;
  // sort work
  int* key;         // global cell key of slot
  int* slot;        // position inside the cell from the atomic histogram
  int* cell_count;  // total_cells + 1
  int* cell_start;  // total_cells + 1
  int* tmp_src;     // unstable placement: source slot
  int* tmp_id;      // unstable placement: caller index
  int* tmp_key;
  // outputs of the fine-grained calls
  double4* ACC;     // dv/dt
  double* DDEN;     // drho/dt
  double* MSUM;     // FP32c momentum pair sums of a slot: 9 values (pressure, Monaghan, Morris x 3)
  float4* VF2;      // FP32c with velocity smoothing: the step's leapfrog velocities in FP32
  double* BG;      // with C1: B_ren_gradp, B(i,j) at [(3 i + j) total_slots + slot]
  double* BD;      // with C1_divu: B_ren_divu, same layout
  // removal replay
  uint8_t* out_flag;   // by caller index
  int* id_remap;       // by caller index
  int* cur_of;
  int total_cells;
  int total_slots;
};

__host__ __device__ inline int cell_key_local(const SimDev& s, int i, int j, int k) {
  return ((j - 1) * s.ncd[0] + (i - 1)) * s.ncd[2] + (k - 1);
}

}  // namespace sph
