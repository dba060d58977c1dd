// Device kernels of the FP64 path: cell binning and sort, SA-SPH boundary
// data, continuity and momentum pair passes, leapfrog, EoS and time step.
//
// Compiled with --fmad=false: every FP64 expression below is evaluated in
// the reference's left-to-right order without contraction, like the
// gfortran -O2 x86-64 build of the reference (src/Makefile:124), so the
// pair sums reproduce the reference's rounding.
#include <cstdint>
#include <cfloat>
#include "../../include/sphera_b200.h"
#include "sph_internal.cuh"
#include "sph_launch.h"

namespace sph {

// BoundIntegralTab2D (SA_SPH_module.f90:29-54), filled by the host with the
// single-precision roundings of the table's default-REAL literals.
__constant__ double c_bit2d[22][6];

namespace {

constexpr double kMaxPositive = 3.4e+38;       // max_positive_number
constexpr double kPigreco = 3.14159265358979e0;
constexpr double kKernelConst2D = 0.454728408833987e0;
constexpr double kDeltaXBit = 0.1;

// --------------------------------------------------------------------------
// small helpers
// --------------------------------------------------------------------------

__device__ __forceinline__ void load_sim(SimDev& dst, const SimDev* src, int sim, int& cur) {
  if (cur == sim) return;
  __syncthreads();
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src + sim);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
  constexpr int n = sizeof(SimDev) / 8;
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
  cur = sim;
  __syncthreads();
}

// ParticleCellNumber.f90:52-62 + CellNumber.f90:53-59: 1-based (i,j,k),
// false if outside the grid.
// a / b rounded to nearest, bit for bit what the IEEE division a / b gives,
// from y = RN(1/b) (a constant's reciprocal formed on the host, or
// __drcp_rn(b) once for a divisor that several divisions share).  The
// method is Markstein's (P. Markstein, IBM J. Res. Dev. 34(1), 1990; the
// theorem in Muller et al., Handbook of Floating-Point Arithmetic, on
// division with a fused multiply-add): if y is within half an ulp of 1/b
// and q within one ulp of a/b, the remainder r = a - b q is exact and
// RN(q + r y) = RN(a/b).  q0 = RN(a y) can be up to 1.5 ulp off, so one
// correction first brings it within half an ulp plus O(2^-105) relative
// (q1), and the second is the theorem's step.  A zero remainder means the
// current q is the exact quotient and is kept as it is (so a zero a keeps
// its sign, which q + 0 y would lose).  Domain: a, b finite, b != 0, and no
// quotient or remainder in the subnormal range -- true of every caller
// (lengths, densities and smoothing lengths of a physical state).
__device__ __forceinline__ double div_rn(double a, double b, double y) {
  const double q0 = __dmul_rn(a, y);
  const double r0 = __fma_rn(-b, q0, a);
  const double q1 = r0 == 0.0 ? q0 : __fma_rn(r0, y, q0);
  const double r1 = __fma_rn(-b, q1, a);
  return r1 == 0.0 ? q1 : __fma_rn(r1, y, q1);
}

__device__ __forceinline__ bool particle_cell(const SimDev& s, double x, double y, double z, int& i, int& j,
                                              int& k) {
  double ci = ceil(div_rn(x - s.extr_lo[0], s.dcd[0], s.rcp_dcd[0])) - (double)s.ioff;   // exact: whole numbers
  double ck = ceil(div_rn(z - s.extr_lo[2], s.dcd[2], s.rcp_dcd[2]));
  double cj = (s.dim == 3) ? ceil(div_rn(y - s.extr_lo[1], s.dcd[1], s.rcp_dcd[1])) : 1.0;
  if (!(ci >= 1.0 && ci <= (double)s.ncd[0] && cj >= 1.0 && cj <= (double)s.ncd[1] && ck >= 1.0 &&
        ck <= (double)s.ncd[2]))
    return false;
  i = (int)ci;
  j = (int)cj;
  k = (int)ck;
  return true;
}

// FP32 offset of a particle from the origin of its cell; w holds the cell's
// k index as a float (exact: k < 2^24), so cell differences are FP32
// subtractions, exact, with no integer-to-float conversion in the pair loops.
__device__ __forceinline__ float4 screening_copy(const SimDev& s, const double4& x) {
  int i, j, k;
  if (!particle_cell(s, x.x, x.y, x.z, i, j, k)) return make_float4(0.f, 0.f, 0.f, -8.0f);
  double ox = s.extr_lo[0] + s.dcd[0] * (i + s.ioff - 1);
  double oy = (s.dim == 3) ? s.extr_lo[1] + s.dcd[1] * (j - 1) : 0.0;
  double oz = s.extr_lo[2] + s.dcd[2] * (k - 1);
  return make_float4((float)(x.x - ox), (float)(x.y - oy), (float)(x.z - oz), (float)k);
}

// Contiguous slot range of neighbour column r (reference order: y, then x).
template <int DIM>
__device__ __forceinline__ void neighbour_run(const SimDev& s, const int* __restrict__ cell_start, int ci, int cj,
                                              int ck, int r, int& b, int& e) {
  int jr = (DIM == 3) ? cj - 1 + r / 3 : cj;
  int ir = ci - 1 + ((DIM == 3) ? r % 3 : r);
  b = 0;
  e = 0;
  if (ir < 1 || ir > s.ncd[0] || jr < 1 || jr > s.ncd[1]) return;
  int klo = ck > 1 ? ck - 1 : 1;
  int khi = ck < s.ncd[2] ? ck + 1 : s.ncd[2];
  int base = s.cell_off + ((jr - 1) * s.ncd[0] + (ir - 1)) * s.ncd[2];
  b = __ldg(cell_start + base + klo - 1);
  e = __ldg(cell_start + base + khi);
}

// Kernel values of CalcVarLength.f90:242-269 for an accepted pair.
__device__ __forceinline__ void kernel_values(const SimDev& s, double rijtemp2, double& PK1, double& PK2,
                                              double& PK3) {
  double rijtemp = sqrt(rijtemp2);
  double rij_su_h = div_rn(rijtemp, s.h, s.rcp_h);
  double rij_su_h_quad = div_rn(rijtemp2, s.squareh, s.rcp_squareh);
  int index_rij_su_h = (int)rij_su_h;
  double denom = 1.0 / (rijtemp + s.eta);
  PK1 = 0.0;
  PK2 = 0.0;
  PK3 = 0.0;
  if (index_rij_su_h >= 2) return;
  double gradmod = -(2.0 * rij_su_h) + 1.5 * rij_su_h_quad;
  double gradmodwacl = -12.0 - 3.0 * rij_su_h_quad + 12.0 * rij_su_h;
  if (index_rij_su_h > 0) gradmod = -gradmod + rij_su_h_quad - 2.0;
  gradmod = gradmod * s.ke_coef;
  gradmodwacl = gradmodwacl * s.kacl_coef;
  PK1 = gradmod * denom;
  PK2 = PK1 / (rijtemp2 + s.eta2);
  PK3 = gradmodwacl * denom;
}

__device__ __forceinline__ void set_status(SimDyn* d, int code) { atomicCAS(&d->status, 0, code); }

__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max(int v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Adds two per-thread counts of the block to counters[0..1] (one atomic per
// block and counter).
__device__ __forceinline__ void block_count2(unsigned long long* counters, int a, int c) {
  unsigned long long sa = (unsigned long long)a, sc = (unsigned long long)c;
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_xor_sync(0xffffffffu, sa, o);
    sc += __shfl_xor_sync(0xffffffffu, sc, o);
  }
  if ((threadIdx.x & 31) == 0 && (sa | sc)) {
    atomicAdd(counters, sa);
    atomicAdd(counters + 1, sc);
  }
}

// InterpolateTable.f90:58-82 on columns 1..4.
__device__ __forceinline__ void interpolate_table(const SimDev& s, double xval, double* iv) {
  double deltaX = s.ktdelta;
  double xval0 = s.kerneltab[0][0];
  int nr0 = (int)div_rn(xval - xval0, deltaX, s.rcp_ktdelta);
  if (nr0 <= 0) {
    for (int c = 0; c < 4; ++c) iv[c] = s.kerneltab[0][c + 1];
  } else if (nr0 >= kKtRows) {
    for (int c = 0; c < 4; ++c) iv[c] = s.kerneltab[kKtRows][c + 1];
  } else {
    double csi = div_rn(xval - s.kerneltab[nr0][0], deltaX, s.rcp_ktdelta);
    for (int c = 0; c < 4; ++c)
      iv[c] = s.kerneltab[nr0][c + 1] + csi * (s.kerneltab[nr0 + 1][c + 1] - s.kerneltab[nr0][c + 1]);
  }
}

// LocalNormalCoordinates.f90:59-87 + IsPointInternal.f90:54-72.
__device__ __forceinline__ bool point_internal(const FaceDev& f, double px, double py) {
  double c0 = (f.AA[0] + f.BB[0] * px + f.CC[0] * py) * f.usu_due_area;
  double c1 = (f.AA[1] + f.BB[1] * px + f.CC[1] * py) * f.usu_due_area;
  if (f.fkod == 2) return !(c0 < 0.0 || c0 > 1.0 || c1 < 0.0 || c1 > 1.0);
  if (f.fkod == 1) {
    double c2 = 1.0 - (c0 + c1);
    return !(c0 < 0.0 || c0 > 1.0 || c1 < 0.0 || c1 > 1.0 || c2 < 0.0 || c2 > 1.0);
  }
  return false;
}

// w.f90:48-57
__device__ __forceinline__ double w_kernel(double r, double h, double coef) {
  double s = r / h, q;
  if (s <= 1.0) q = 0.666666667 + s * s * (s * 0.5 - 1.0);
  else if (s >= 2.0) q = 0.0;
  else {
    double dms = 2.0 - s;
    q = dms * dms * dms / 6.0;
  }
  return q * coef;
}

// WIntegr.f90:57-74
__device__ __forceinline__ double w_integr(double ri, double hh) {
  double ro = ri / hh;
  if (0.0 <= ro && ro < 1.0) {
    double ro2 = ro * ro, ro3 = ro2 * ro;
    double W1 = (0.5 + -0.375 * ro2 + 0.15 * ro3) * ro2;
    return kKernelConst2D * (0.35 - W1);
  } else if (1.0 <= ro && ro < 2.0) {
    double q1 = 2.0 - ro, q2 = q1 * q1, q4 = q2 * q2;
    double W2 = (-0.125 + 0.05 * q1) * q4;
    return -kKernelConst2D * W2;
  }
  return 0.0;
}

// J2Wro2.f90:50-63
__device__ __forceinline__ double j2_wro2(double ro) {
  const double a1 = 0.00833333333333333, a2 = 0.26666666666666667;
  double ro2 = ro * ro, ro3 = ro2 * ro;
  if (0.0 <= ro && ro < 1.0) return kKernelConst2D * (0.25 - (a1 * (40.0 - 36.0 * ro2 + 15.0 * ro3) * ro3));
  if (1.0 <= ro && ro < 2.0)
    return kKernelConst2D * (a2 - (a1 * (80.0 - 90.0 * ro + 36.0 * ro2 - 5.0 * ro3) * ro3));
  return 0.0;
}

// InterpolateBoundaryIntegrals2D.f90:61-69
__device__ __forceinline__ void interp_bit2d(int ncols, const int* col, double xx, double* func) {
  if (xx < c_bit2d[0][0]) xx = c_bit2d[0][0];
  int ii = (int)((xx - c_bit2d[0][0]) / kDeltaXBit) + 1;
  if (ii > 21) ii = 21;  // the table ends at 2.001; deltai < 2 on this path
  double xi = c_bit2d[ii - 1][0];
  for (int nc = 0; nc < ncols; ++nc) {
    double fi = c_bit2d[ii - 1][col[nc]];
    double fip1 = c_bit2d[ii][col[nc]];
    func[nc] = fi + (fip1 - fi) * (xx - xi) / kDeltaXBit;
  }
}

}  // namespace

// ==========================================================================
// Sorting (OrdGrid1 replacement)
// ==========================================================================

// Copies the sorted state into the scratch record the sort consumes.
__global__ void k_stage(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count) continue;
    const Particles& P = b.P;
    double4 x = P.X[p];
    double4 v = P.V[p];
    double2 rp = P.RP[p];
    P.X2[p] = x;
    P.V2[p] = make_double4(v.x, v.y, v.z, rp.x);
    P.P2[p] = rp.y;
    P.I2[p] = P.I[p];
    P.L2[p] = P.L[p];
  }
}

// Cell key of every slot + atomic histogram.  KeyKind::Sort bins the
// scratch record by the z-fastest layout key; KeyKind::Reference bins the
// sorted state by CellNumber.f90's numbering for the grid dump.
template <KeyKind KIND>
__global__ void k_bin(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  const int lane = threadIdx.x & 31;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    const bool valid = threadIdx.x < tl.count;
    int p = tl.start + threadIdx.x;
    int key = -1;
    if (valid) {
      SimDyn* dyn = b.dyn + tl.sim;
      int nag = dyn->nag;
      key = s.cell_off + s.ncells;  // removal bin
      if (p < s.p_off + nag) {
        double4 x = (KIND == KeyKind::Sort) ? P.X2[p] : P.X[p];
        int i, j, k;
        if (particle_cell(s, x.x, x.y, x.z, i, j, k)) {
          key = s.cell_off + ((KIND == KeyKind::Sort) ? cell_key_local(s, i, j, k)
                                                       : ((k - 1) * s.ncd[1] + (j - 1)) * s.ncd[0] + (i - 1));
        } else if (KIND == KeyKind::Sort) {
          atomicAdd(&dyn->n_out, 1);
          P.out_flag[s.p_off + P.I2[p] - 1] = 1;
        }
      }
      P.key[p] = key;
    }
    // the lanes of a warp that bin into one cell (the last sort's order
    // keeps most of a warp in one or two) take their slots with one atomic;
    // a slot only has to be unique within its cell (the placement is ranked
    // by caller index afterwards)
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (valid && lane == leader) base = atomicAdd(P.cell_count + key, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (valid) P.slot[p] = base + __popc(peers & ((1u << lane) - 1u));
  }
}

// OrdGrid1.f90:58-82: particles out of the grid are removed by moving the
// last particle into their place, in increasing particle index.  Replayed
// exactly (one thread per simulation, only when a removal happened).
__global__ void k_removal(DevBatch b) {
  int sim = blockIdx.x;
  if (threadIdx.x != 0 || sim >= b.nsims) return;
  SimDyn* d = b.dyn + sim;
  if (d->n_out == 0) return;
  const SimDev& s = b.sims[sim];
  uint8_t* out = b.P.out_flag + s.p_off - 1;   // 1-based by caller index
  int* cur_of = b.P.cur_of + s.p_off - 1;
  int* remap = b.P.id_remap + s.p_off - 1;
  int n0 = d->nag;
  int n = n0;
  for (int id = 1; id <= n0; ++id) { cur_of[id] = id; remap[id] = 0; }
  int npi = 0;
  while (n > 0 && npi < n) {
    npi = npi + 1;
    if (out[npi]) {
      out[npi] = out[n];
      cur_of[npi] = cur_of[n];
      n = n - 1;
      npi = npi - 1;
    }
  }
  for (int id = 1; id <= n; ++id) remap[cur_of[id]] = id;
  for (int id = 1; id <= n0; ++id) out[id] = 0;
  d->removed_total += n0 - n;
  d->nag = n;
  d->warnings |= SPH_WARN_PARTICLES_REMOVED;
}

// Exclusive scan of the cell histogram (3 phases), clearing the histogram.
__device__ __forceinline__ int block_excl_scan(int v, int* warp_sums, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int ws = lane < nw ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    if (lane < nw) warp_sums[lane] = ws;
  }
  __syncthreads();
  int base = wid > 0 ? warp_sums[wid - 1] : 0;
  total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanChunk = kScanThreads * kScanPer;

__global__ void __launch_bounds__(kScanThreads) k_scan1(const int* __restrict__ cnt, int n, int* block_sums) {
  __shared__ int ws[32];
  int base = blockIdx.x * kScanChunk + threadIdx.x * kScanPer;
  int v = 0;
  for (int q = 0; q < kScanPer; ++q) v += (base + q < n) ? cnt[base + q] : 0;
  int total;
  block_excl_scan(v, ws, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan2(int* block_sums, int nb, int* cell_start, int n) {
  __shared__ int ws[32];
  int carry = 0;
  for (int c0 = 0; c0 < nb; c0 += kScanThreads) {
    int i = c0 + threadIdx.x;
    int v = i < nb ? block_sums[i] : 0;
    int total;
    int ex = block_excl_scan(v, ws, total);
    if (i < nb) block_sums[i] = ex + carry;
    carry += total;
  }
  if (threadIdx.x == 0) cell_start[n] = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_scan3(int* cnt, int n, const int* block_sums, int* cell_start) {
  __shared__ int ws[32];
  int base = blockIdx.x * kScanChunk + threadIdx.x * kScanPer;
  int vals[kScanPer];
  int v = 0;
  for (int q = 0; q < kScanPer; ++q) {
    vals[q] = (base + q < n) ? cnt[base + q] : 0;
    v += vals[q];
  }
  int total;
  int ex = block_excl_scan(v, ws, total) + block_sums[blockIdx.x];
  for (int q = 0; q < kScanPer; ++q) {
    if (base + q < n) {
      cell_start[base + q] = ex;
      cnt[base + q] = 0;
    }
    ex += vals[q];
  }
}

// Unstable placement by cell (the atomic slot), remembering the source.
__global__ void k_place(DevBatch b, const int* __restrict__ cstart, int use_scratch_ids) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int p = tl.start + threadIdx.x;
    int key = P.key[p];
    int dst = cstart[key] + P.slot[p];
    int id = use_scratch_ids ? P.I2[p] : P.I[p];
    if (use_scratch_ids && b.dyn[tl.sim].n_out > 0 && id > 0) id = P.id_remap[s.p_off + id - 1];
    P.tmp_src[dst] = p;
    P.tmp_id[dst] = id;
    P.tmp_key[dst] = key;
  }
}

// Rank inside the cell by caller index (OrdGrid1.f90:100-105 stable
// scatter) and gather the scratch record into the sorted state.
// PART selects what is gathered: kPermuteAll everything (the step); the IC
// of an upload splits it in two so that the velocities, densities and
// pressures can still be on their way from the host while the lists and
// the boundary data are built from the sorted positions:
// kPermutePositions gathers x, m, the caller index and the laminar flag and
// keeps each slot's destination in P.slot (free once k_place has run);
// kPermuteRest gathers the rest through it.
constexpr int kPermuteAll = 0, kPermutePositions = 1, kPermuteRest = 2;

template <int PART>
__global__ void k_rank_permute(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int d = tl.start + threadIdx.x;
    int fin = d;
    if (PART == kPermuteRest) {
      fin = P.slot[d];
    } else {
      int key = P.tmp_key[d];
      int myid = P.tmp_id[d];
      if (key != s.cell_off + s.ncells) {
        int cs = P.cell_start[key], ce = P.cell_start[key + 1];
        int rank = 0;
        for (int q = cs; q < ce; ++q) rank += (P.tmp_id[q] < myid) ? 1 : 0;
        fin = cs + rank;
      }
      P.I[fin] = myid;
      if (PART == kPermutePositions) P.slot[d] = fin;
    }
    int src = P.tmp_src[d];
    double4 x = P.X2[src];
    if (PART != kPermuteRest) {
      P.X[fin] = x;
      P.XF[fin] = screening_copy(s, x);
      P.L[fin] = P.L2[src];
    }
    if (PART != kPermutePositions) {
      double4 v = P.V2[src];
      double vol = x.w / v.w;
      double pr = P.P2[src];
      P.V[fin] = make_double4(v.x, v.y, v.z, vol);
      P.RP[fin] = make_double2(v.w, pr);
      P.VF[fin] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)vol);
      P.RF[fin] = make_float4((float)v.w, (float)(pr / (v.w * v.w)), (float)x.w, 0.f);
      P.RM[fin] = make_float2((float)v.w, (float)(pr / (v.w * v.w)));
    }
  }
}

// NPartOrd of the reference numbering (verification only).
__global__ void k_rank_reference(DevBatch b, const int* __restrict__ cstart, int* npartord) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int d = tl.start + threadIdx.x;
    int key = P.tmp_key[d];
    if (key == s.cell_off + s.ncells) continue;
    int myid = P.tmp_id[d];
    int cs = cstart[key], ce = cstart[key + 1];
    int rank = 0;
    for (int q = cs; q < ce; ++q) rank += (P.tmp_id[q] < myid) ? 1 : 0;
    npartord[cs + rank - s.p_off] = myid;
  }
}

// ==========================================================================
// SA-SPH boundary data (ComputeBoundaryDataTab_3D / _2D)
// ==========================================================================

// ComputeBoundaryVolumeIntegrals_P0.f90:81-155 for one (particle, face).
// The point-in-face test of one face held in registers (the same arithmetic
// as point_internal).
struct FaceTest {
  double a0, a1, b0, b1, c0, c1, u;
  int fkod;
  __device__ __forceinline__ void load(const FaceDev& f) {
    a0 = f.AA[0];
    a1 = f.AA[1];
    b0 = f.BB[0];
    b1 = f.BB[1];
    c0 = f.CC[0];
    c1 = f.CC[1];
    u = f.usu_due_area;
    fkod = f.fkod;
  }
  __device__ __forceinline__ bool inside(double px, double py) const {
    double k0 = (a0 + b0 * px + c0 * py) * u;
    double k1 = (a1 + b1 * px + c1 * py) * u;
    if (fkod == 2) return !(k0 < 0.0 || k0 > 1.0 || k1 < 0.0 || k1 > 1.0);
    if (fkod == 1) {
      double k2 = 1.0 - (k0 + k1);
      return !(k0 < 0.0 || k0 > 1.0 || k1 < 0.0 || k1 > 1.0 || k2 < 0.0 || k2 > 1.0);
    }
    return false;
  }
};

__device__ void face_integrals(const SimDev& s, const double* __restrict__ bit, const FaceDev& f,
                               const double* locx, BdtEntry& e) {
  FaceTest ft;
  ft.load(f);
  double IntWdV = 0.0, IntdWrm1dV = 0.0, IntGWZrm1dV = 0.0;
  double G0 = 0.0, G1 = 0.0, G2 = 0.0;
  double R00 = 0.0, R01 = 0.0, R02 = 0.0, R11 = 0.0, R12 = 0.0, R22 = 0.0;
  double J0 = 0.0, J1 = 0.0, J2 = 0.0, J3 = 0.0;
  double L0 = locx[0], L1 = locx[1], L2 = locx[2];
  if (!(L2 < 0.0)) {
    if (L2 < s.zpmin) L2 = s.zpmin;
    double robpre = 2.1;
    for (int ring = 0; ring < 8; ++ring) {
      const double* row0 = bit + ring * 32 * 7;
      double zp = row0[2];
      double lpj2 = L2 + zp;
      if (!(lpj2 <= 0.0)) continue;       // the whole ring lies above the face plane
      double tsegnato = L2 / (L2 - lpj2);
      // The points of a ring share their polar angle, so their distances to
      // the particle differ by rounding only (s.ring_skip bounds that far
      // below 1e-6 in rob).  After the ring's first inside point the
      // refresh test |rob - robpre| > 1e-3 is therefore false for every
      // later point -- unless the first point missed the threshold by less
      // than 1e-6, when the ring is tested point by point.  Skipping the
      // test skips its distance, square root and division.
      bool test_all = !s.ring_skip, first = true;
      for (int q = 0; q < 32; ++q) {
        const double* row = row0 + q * 7;
        double lpj0 = L0 + row[0];
        double lpj1 = L1 + row[1];
        double px0 = L0 + (lpj0 - L0) * tsegnato;
        double px1 = L1 + (lpj1 - L1) * tsegnato;
        if (!ft.inside(px0, px1)) continue;
        if (first || test_all) {
          double d0 = px0 - L0, d1 = px1 - L1, d2 = 0.0 - L2;
          double dist = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
          double rob = div_rn(dist, s.h, s.rcp_h);
          const double gap = fabs(rob - robpre);
          if (first && !(gap > 1.0e-3) && gap > 1.0e-3 - 1.0e-6) test_all = true;
          first = false;
          if (gap > 1.0e-3) {
            double iv[4];
            interpolate_table(s, rob, iv);
            double da = row[3];
            J0 = iv[0] * da;
            J1 = iv[1] * da;
            J2 = iv[2] * da;
            J3 = iv[3] * da;
            robpre = rob;
          }
        }
        double r0 = row[4], r1 = row[5], r2 = row[6];
        double RZ2 = r2 * r2;
        IntWdV = IntWdV + J0;
        IntdWrm1dV = IntdWrm1dV + J1;
        IntGWZrm1dV = IntGWZrm1dV + RZ2 * J1;
        G0 = G0 + r0 * J2;
        R00 = R00 + r0 * r0 * J3;
        R01 = R01 + r0 * r1 * J3;
        R02 = R02 + r0 * r2 * J3;
        G1 = G1 + r1 * J2;
        R11 = R11 + r1 * r1 * J3;
        R12 = R12 + r1 * r2 * J3;
        G2 = G2 + r2 * J2;
        R22 = R22 + r2 * r2 * J3;
      }
    }
    if (L2 == s.zpmin) IntWdV = point_internal(f, L0, L1) ? 0.5 : 0.0;
  }
  e.bi[0] = 0.0;
  e.bi[1] = IntWdV;
  e.bi[2] = IntdWrm1dV;
  e.bi[3] = G0;
  e.bi[4] = G1;
  e.bi[5] = G2;
  e.bi[6] = IntGWZrm1dV;
  e.bi[7] = 0.0;
  e.ig[0] = R00; e.ig[1] = R01; e.ig[2] = R02;
  e.ig[3] = R01; e.ig[4] = R11; e.ig[5] = R12;
  e.ig[6] = R02; e.ig[7] = R12; e.ig[8] = R22;
}

// ComputeBoundaryDataTab_3D.f90:67-105 with FindCloseBoundaryFaces3D.f90:79-188.
__global__ void __launch_bounds__(kBlock) k_boundary3d(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int p = tl.start + threadIdx.x;
    SimDyn* dyn = b.dyn + tl.sim;
    P.bdt_count[p] = 0;
    if (p >= s.p_off + dyn->nag || s.nfaces == 0) continue;
    double4 x = P.X[p];
    int ic, jc, kc;
    if (!particle_cell(s, x.x, x.y, x.z, ic, jc, kc)) continue;
    if (!b.cell_near[s.cell_off + cell_key_local(s, ic, jc, kc)]) continue;
    int clob[kMaxLocalFaces];
    double pin[kMaxLocalFaces];
    int ncbf = 0;
    bool overflow = false;
    for (int i = ic - 1; i <= ic + 1; ++i)
      for (int j = jc - 1; j <= jc + 1; ++j)
        for (int k = kc - 1; k <= kc + 1; ++k) {
          if (i < 1 || i > s.ncd[0] || j < 1 || j > s.ncd[1] || k < 1 || k > s.ncd[2]) continue;
          int gk = s.cell_off + cell_key_local(s, i, j, k);
          int nf = b.cf_count[gk];
          int fs = b.cf_start[gk];
          for (int q = 0; q < nf; ++q) {
            int fid = b.cf_list[fs + q];
            bool there = false;
            for (int u = 0; u < ncbf && u < kMaxLocalFaces; ++u) there |= (clob[u] == fid);
            if (there) continue;
            const FaceDev& f = b.faces[s.face_off + fid - 1];
            double pn = 0.0;
            pn = pn + f.T[0][2] * (x.x - f.GXref[0]);
            pn = pn + f.T[1][2] * (x.y - f.GXref[1]);
            pn = pn + f.T[2][2] * (x.z - f.GXref[2]);
            if (pn >= 0.0 && pn < s.doubleh) {
              if (ncbf >= s.maxcb || ncbf >= kMaxLocalFaces) {
                overflow = true;
              } else {
                clob[ncbf] = fid;
                pin[ncbf] = pn;
              }
              ncbf++;
            }
          }
        }
    if (overflow) {
      set_status(dyn, SPH_ERR_CLOSE_FACES);
      continue;
    }
    if (ncbf == 0) continue;
    // each simulation draws on its own quota of the shared pool first, so
    // one that overflows fails alone and the others' entries are unaffected
    if (atomicAdd(&dyn->bdt_sim_used, ncbf) + ncbf > s.bdt_quota) {
      set_status(dyn, SPH_ERR_BDT_OVERFLOW);
      continue;
    }
    int gbase = atomicAdd(&b.dyn[b.nsims].bdt_used, ncbf);  // global allocation counter
    if (gbase + ncbf > P.bdt_cap) {
      set_status(dyn, SPH_ERR_BDT_OVERFLOW);
      continue;
    }
    atomicMax(&dyn->ncbf_max, ncbf);
    P.bdt_count[p] = ncbf;
    P.bdt_start[p] = gbase;
    for (int u = 0; u < ncbf; ++u) {
      const FaceDev& f = b.faces[s.face_off + clob[u] - 1];
      double locx[3];
      for (int sdi = 0; sdi < 2; ++sdi) {
        double acc = 0.0;
        acc = acc + f.T[0][sdi] * (x.x - f.GXref[0]);
        acc = acc + f.T[1][sdi] * (x.y - f.GXref[1]);
        acc = acc + f.T[2][sdi] * (x.z - f.GXref[2]);
        locx[sdi] = acc;
      }
      locx[2] = pin[u];
      BdtEntry& e = P.bdt[gbase + u];
      e.loc[0] = locx[0];
      e.loc[1] = locx[1];
      e.loc[2] = locx[2];
      e.clobonum = clob[u];
      e.pad = tl.sim;            // the integrals pass needs the simulation
    }
  }
}

// ComputeBoundaryVolumeIntegrals_P0.f90:81-155 for every entry the find
// pass allocated, one (particle, face) per thread: the quadrature costs are
// balanced across the GPU whatever the particles' distribution over tiles.
__global__ void __launch_bounds__(128) k_boundary3d_integrals(DevBatch b) {
  // the simulation constants and hemisphere table of the chunk's first
  // entry, staged in shared memory (a batch chunk can mix simulations:
  // entries of another one read theirs from global memory)
  __shared__ SimDev ssim;
  __shared__ double sbit[kBitRows * 7];
  int loaded = -1;
  int used = b.dyn[b.nsims].bdt_used;
  if (used > b.P.bdt_cap) used = b.P.bdt_cap;
  for (int base = blockIdx.x * blockDim.x; base < used; base += gridDim.x * blockDim.x) {
    const int first = b.P.bdt[base].pad;
    if (first != loaded) {
      load_sim(ssim, b.sims, first, loaded);
      const double* src = b.bit + (size_t)first * kBitRows * 7;
      for (int i = threadIdx.x; i < kBitRows * 7; i += blockDim.x) sbit[i] = src[i];
      __syncthreads();
    }
    const int idx = base + threadIdx.x;
    if (idx >= used) continue;
    BdtEntry& e = b.P.bdt[idx];
    const int sim = e.pad;
    const bool mine = sim == loaded;
    const SimDev& s = mine ? ssim : b.sims[sim];
    const double* bit = mine ? sbit : b.bit + (size_t)sim * kBitRows * 7;
    const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
    double locx[3] = {e.loc[0], e.loc[1], e.loc[2]};
    BdtEntry r;
    face_integrals(s, bit, f, locx, r);
    for (int q = 0; q < 8; ++q) e.bi[q] = r.bi[q];
    for (int q = 0; q < 9; ++q) e.ig[q] = r.ig[q];
  }
}

// ComputeBoundaryDataTab_2D.f90:70-157 with FindCloseBoundarySides2D,
// SelectCloseBoundarySides2D, FindBoundaryIntersection2D,
// ComputeSurfaceIntegral_WdS2D, BoundaryVolumeIntegrals2D,
// ComputeVolumeIntegral_WdV2D and InterpolateBoundaryIntegrals2D.
__global__ void __launch_bounds__(kBlock) k_boundary2d(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int p = tl.start + threadIdx.x;
    SimDyn* dyn = b.dyn + tl.sim;
    P.bdt_count[p] = 0;
    if (p >= s.p_off + dyn->nag || s.nsides == 0) continue;
    double4 x = P.X[p];
    const SideDev* sd = b.sides + s.side_off;
    int clob[kMaxCloseSides];
    double lx[kMaxCloseSides], ly[kMaxCloseSides];
    int ncbs = 0;
    bool overflow = false;
    for (int isi = 1; isi <= s.nsides; ++isi) {
      const SideDev& S = sd[isi - 1];
      double P1P0 = x.x - S.v1[0], P1P1 = x.z - S.v1[1];
      double sidel = S.length;
      double xp = P1P0 * S.sss[0] + P1P1 * S.sss[1];
      double yp = P1P0 * S.nnn[0] + P1P1 * S.nnn[1];
      double xpmin = -s.doubleh, xpmax = sidel + s.doubleh;
      double ypmin = -s.doubleh, ypmax = s.doubleh;
      if ((xpmin < xp && xp < xpmax) && (ypmin < yp && yp < ypmax)) {
        double ypmx = 0.0, ypmn = 0.0;
        if (xp < 0.0) {
          ypmx = sqrt(s.square_doubleh - xp * xp);
          ypmn = -ypmx;
        } else if (xp <= sidel) {
          ypmx = ypmax;
          ypmn = ypmin;
        } else if (xp < xpmax) {
          double L = (sidel - xp) * (sidel - xp);
          ypmx = sqrt(s.square_doubleh - L);
          ypmn = -ypmx;
        }
        if (ypmn < yp && yp < ypmx) {
          if (ncbs >= kMaxCloseSides) {
            overflow = true;
          } else {
            clob[ncbs] = isi;
            lx[ncbs] = xp;
            ly[ncbs] = yp;
          }
          ncbs++;
        }
      }
    }
    if (overflow) {
      set_status(dyn, SPH_ERR_CLOSE_SIDES);
      continue;
    }
    if (ncbs == 0) continue;
    if (ncbs == 2) {
      if (sd[clob[0] - 1].previous_side == clob[1]) lx[1] = sd[clob[1] - 1].length - lx[1];
      else if (sd[clob[1] - 1].previous_side == clob[0]) lx[0] = sd[clob[0] - 1].length - lx[0];
    }
    // SelectCloseBoundarySides2D: fixe / tapi sides in front of the particle
    int ib[kMaxCloseSides];
    double ix[kMaxCloseSides], iy[kMaxCloseSides];
    int nint = 0;
    for (int c = 0; c < ncbs; ++c)
      if (ly[c] > 0.0) {
        ib[nint] = clob[c];
        ix[nint] = lx[c];
        iy[nint] = ly[c];
        nint++;
      }
    if (nint == 0) continue;
    if (atomicAdd(&dyn->bdt_sim_used, nint) + nint > s.bdt_quota) {
      set_status(dyn, SPH_ERR_BDT_OVERFLOW);
      continue;
    }
    int gbase = atomicAdd(&b.dyn[b.nsims].bdt_used, nint);
    if (gbase + nint > P.bdt_cap) {
      set_status(dyn, SPH_ERR_BDT_OVERFLOW);
      continue;
    }
    P.bdt_count[p] = nint;
    P.bdt_start[p] = gbase;
    for (int c = 0; c < nint; ++c) {
      BdtEntry e;
      for (int q = 0; q < 9; ++q) e.ig[q] = 0.0;
      for (int q = 0; q < 8; ++q) e.bi[q] = 0.0;
      e.clobonum = ib[c];
      e.pad = 0;
      e.loc[0] = ix[c];
      e.loc[1] = iy[c];
      e.loc[2] = 0.0;
      double func[5] = {0, 0, 0, 0, 0};
      if (nint == 2) {
        // FindBoundaryIntersection2D.f90:61-92
        double minlen = 0.01 * s.h;
        double xpi = ix[c], ypi = iy[c];
        if (ypi < 0.0) ypi = 0.0;
        double halfchord = sqrt(s.square_doubleh - ypi * ypi);
        double XA = xpi - halfchord, XB = xpi + halfchord;
        double xpmin = 0.0;
        if (XA > xpmin) xpmin = XA;
        double xpmax = sd[ib[c] - 1].length;
        if (XB < xpmax) xpmax = XB;
        double interlen = xpmax - xpmin;
        if (interlen <= minlen) interlen = 0.0;
        // ComputeSurfaceIntegral_WdS2D.f90:57-83
        double IntWdS = 0.0;
        if (interlen > 0.0) {
          double dsrif = s.h / 2;
          double ypc = iy[c] < 0.0 ? 0.0 : iy[c];
          double ypiq = ypc * ypc;
          int ndiv = (int)(interlen / dsrif + 0.5);
          if (ndiv < 2) ndiv = 2;
          double deltas = interlen / ndiv;
          double xpip = xpmin - 0.5 * deltas;
          for (int ipt = 1; ipt <= ndiv; ++ipt) {
            xpip = xpip + deltas;
            double dxpip = xpip - ix[c];
            double ris = sqrt(dxpip * dxpip + ypiq);
            IntWdS = IntWdS + w_kernel(ris, s.h, s.coefke) * deltas;
          }
        }
        // BoundaryVolumeIntegrals2D.f90
        double IntWdV = 0.0, D0 = 0.0, D1 = 0.0;
        double dalfarif = kPigreco / 10;
        double yplimite = 0.05 * s.h;
        if (interlen > 0.0) {
          double ypb = iy[c];
          if (ypb < yplimite) ypb = yplimite;
          double alfaA = atan2(xpmin - ix[c], ypb), alfaB = atan2(xpmax - ix[c], ypb);
          double Intalfa = alfaB - alfaA;
          int ndiv = (int)(Intalfa / dalfarif + 0.5);
          if (ndiv < 1) ndiv = 1;
          double dalfa = Intalfa / ndiv;
          double alfa_k = alfaA - 0.5 * dalfa;
          for (int k = 1; k <= ndiv; ++k) {
            alfa_k = alfa_k + dalfa;
            double sa = sin(alfa_k), ca = cos(alfa_k);
            double rb = ypb / ca;
            double rob = div_rn(rb, s.h, s.rcp_h);
            double mult = s.h * j2_wro2(rob) * dalfa;
            D0 = D0 + sa * mult;
            D1 = D1 - ca * mult;
            IntWdV = IntWdV + w_integr(rb, s.h) * dalfa;
          }
          if (ypb == yplimite) IntWdV = 0.5;
        }
        // ComputeVolumeIntegral_WdV2D.f90
        double IntWdV1 = 0.0;
        if (interlen > 0.0) {
          double ypv = iy[c];
          if (ypv >= yplimite) {
            double alfaA = atan2(xpmin - ix[c], ypv), alfaB = atan2(xpmax - ix[c], ypv);
            double Intalfa = alfaB - alfaA;
            int ndiv = (int)(Intalfa / dalfarif + 0.5);
            if (ndiv < 2) ndiv = 2;
            double dalfa = Intalfa / ndiv;
            double alfa = alfaA - 0.5 * dalfa;
            for (int ipt = 1; ipt <= ndiv; ++ipt) {
              alfa = alfa + dalfa;
              double ta = tan(alfa);
              double ris = ypv * sqrt(1.0 + ta * ta);
              IntWdV1 = IntWdV1 + w_integr(ris, s.h) * dalfa;
            }
          } else {
            int jc = 1 - c;  // the other side (nint == 2)
            double ypj = iy[jc];
            if (ypj <= yplimite) {
              double angle = 0.0;
              if (sd[ib[0] - 1].previous_side == ib[1]) angle = sd[ib[0] - 1].angle;
              else if (sd[ib[1] - 1].previous_side == ib[0]) angle = sd[ib[1] - 1].angle;
              else set_status(dyn, 804);
              IntWdV1 = 0.5 * (angle + kPigreco) / (2.0 * kPigreco);
            } else {
              IntWdV1 = (xpmin >= ix[c] && ix[c] <= xpmax) ? 0.5 : 0.0;
            }
          }
        }
        const int col[3] = {3, 4, 5};
        interp_bit2d(3, col, iy[c] / s.h, func);
        e.bi[0] = IntWdS;
        e.bi[1] = IntWdV;
        e.bi[2] = IntWdV1;
        e.bi[3] = D0;
        e.bi[4] = D1;
        e.bi[5] = func[0] / s.squareh;
        e.bi[6] = func[1] / s.squareh;
        e.bi[7] = func[2] / s.squareh;
      } else if (nint == 1) {
        const int col[5] = {1, 2, 3, 4, 5};
        interp_bit2d(5, col, iy[c] / s.h, func);
        e.bi[0] = func[0] / s.h;
        e.bi[1] = func[1];
        e.bi[2] = func[1];
        e.bi[3] = 0.0;
        e.bi[4] = 0.0;
        e.bi[5] = func[2] / s.squareh;
        e.bi[6] = func[3] / s.squareh;
        e.bi[7] = func[4] / s.squareh;
      }
      P.bdt[gbase + c] = e;
    }
  }
}

// ==========================================================================
// Momentum: RHS_momentum_equation + inter_EqMoto + viscomon + viscomorris
// + AddBoundaryContributions_to_ME3D/2D + AddElasticBoundaryReaction_3D/2D,
// optionally fused with Leapfrog_momentum, velocity_smoothing_2 (TetaV=0),
// Leapfrog_trajectories and the CFL part of time_step_duration.
// ==========================================================================

// ---------------------------------------------------------------------------
// 1st-order consistency (input_any_t%C1_BE, %C1_divu; 3D).  The matrices are
// held as 9 doubles B(i,j) at 3 i + j, component-major over the slots.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_b(const double* __restrict__ src, int total, int p, double* B) {
  for (int k = 0; k < 9; ++k) B[k] = src[(size_t)k * total + p];
}

__device__ __forceinline__ void store_b(double* dst, int total, int p, const double* B) {
  for (int k = 0; k < 9; ++k) dst[(size_t)k * total + p] = B[k];
}

// Matrix_Inversion_3x3.f90:50-74 as B_ren_gradp_inversion.f90:58-74 and
// B_ren_divu_inversion.f90 use it: the inverse where |det| >= the
// threshold, else -I.
__device__ __forceinline__ void b_inversion(double* B, double thresh) {
  const double det = B[0] * B[4] * B[8] + B[3] * B[7] * B[2] + B[6] * B[1] * B[5] - B[0] * B[7] * B[5] -
                     B[6] * B[4] * B[2] - B[3] * B[1] * B[8];
  if (fabs(det) >= thresh) {
    double inv[9];
    inv[0] = B[4] * B[8] - B[5] * B[7];
    inv[1] = B[2] * B[7] - B[1] * B[8];
    inv[2] = B[1] * B[5] - B[2] * B[4];
    inv[3] = B[5] * B[6] - B[3] * B[8];
    inv[4] = B[0] * B[8] - B[2] * B[6];
    inv[5] = B[2] * B[3] - B[0] * B[5];
    inv[6] = B[3] * B[7] - B[4] * B[6];
    inv[7] = B[1] * B[6] - B[0] * B[7];
    inv[8] = B[0] * B[4] - B[1] * B[3];
    for (int k = 0; k < 9; ++k) B[k] = inv[k] / det;
  } else {
    for (int k = 0; k < 9; ++k) B[k] = 0.0;
    B[0] = B[4] = B[8] = -1.0;
  }
}

// v <- -(B v): MatrixProduct.f90 followed by the sign change of
// inter_EqMoto.f90:255-260, AddBoundaryContributions_to_ME3D.f90:320-325,
// SASPH_continuity.f90:126-140 and Continuity_Equation.f90:201-217.
__device__ __forceinline__ void b_renormalise(const double* B, double* v) {
  double a[3];
  for (int i = 0; i < 3; ++i) {
    double sum = 0.0;
    for (int k = 0; k < 3; ++k) sum = sum + B[3 * i + k] * v[k];
    a[i] = sum;
  }
  for (int i = 0; i < 3; ++i) v[i] = -a[i];
}

// The SA-SPH frontier's contribution T (IntGiWrRdV T^T) to the matrices,
// AddBoundaryContributions_to_ME3D.f90:172-187 and
// AddBoundaryContribution_to_CE3D.f90:93-112, added into B.
__device__ __forceinline__ void add_frontier_b(const FaceDev& f, const BdtEntry& e, double* B) {
  double m2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k) sum = sum + e.ig[3 * i + k] * f.T[j][k];
      m2[3 * i + j] = sum;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k) sum = sum + f.T[i][k] * m2[3 * k + j];
      B[3 * i + j] = B[3 * i + j] + sum;
    }
}

// AddBoundaryContributions_to_ME3D.f90:105-336 (fixe/tapi, slip mode 1).
// C1: B is B_ren_gradp; on the first step (first) the frontiers add to it
// and it is inverted here, after the face loop; gradpt is renormalised.
template <bool C1 = false>
__device__ __forceinline__ void me_boundary3d(const SimDev& s, const DevBatch& b, int nb, int start, const double* vi, double rhoi,
                              double pres, int lam, const double* grav, double* tpres, double* tdiss, double* tvisc,
                              double* B = nullptr, bool first = false) {
  double ALEt[3] = {0, 0, 0}, gradpt[3] = {0, 0, 0}, VMon[3] = {0, 0, 0}, VShear[3] = {0, 0, 0};
  for (int u = 0; u < nb; ++u) {
    const BdtEntry& e = b.P.bdt[start + u];
    const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
    if (!(e.loc[2] > 0.0)) continue;
    double dvn = 0.0;
    for (int SD = 0; SD < 3; ++SD) {
      double dvij = 2.0 * (vi[SD] - f.velocity[SD]);
      dvn = dvn + f.T[SD][2] * dvij;
    }
    double gl[3];
    for (int SD = 0; SD < 3; ++SD) {
      double a = 0.0;
      for (int sdj = 0; sdj < 3; ++sdj) a = a + f.T[sdj][SD] * grav[sdj];
      gl[SD] = a;
    }
    double loc[3];
    for (int i = 0; i < 3; ++i) {
      double a = 0.0;
      for (int k = 0; k < 3; ++k) a = a + e.ig[3 * i + k] * gl[k];
      loc[i] = a;
    }
    for (int i = 0; i < 3; ++i) {
      double a = 0.0;
      for (int k = 0; k < 3; ++k) a = a + f.T[i][k] * loc[k];
      gradpt[i] = gradpt[i] + a;
    }
    double aloc[3];
    for (int k = 0; k < 3; ++k) aloc[k] = 2.0 * pres / rhoi * e.bi[3 + k];
    for (int i = 0; i < 3; ++i) {
      double a = 0.0;
      for (int k = 0; k < 3; ++k) a = a + f.T[i][k] * aloc[k];
      ALEt[i] = ALEt[i] + a;
    }
    if (C1 && first) add_frontier_b(f, e, B);
    double IntGWZrm1dV = e.bi[6];
    double IntdWrm1dV = e.bi[2];
    if (s.alfa_mon > 0.0) {
      double Monvisc = s.alfa_mon * s.celerita * s.h;
      double Mmult = -(Monvisc * dvn * IntGWZrm1dV);
      for (int d = 0; d < 3; ++d) VMon[d] = VMon[d] + Mmult * f.T[d][2];
    }
    double cinvisci = s.kin_visc;
    if (cinvisci > 0.0 && (lam == 1 || !f.laminar_no_slip_check)) {
      double cinviscmult = cinvisci * IntdWrm1dV * f.slip;
      for (int d = 0; d < 3; ++d) VShear[d] = VShear[d] + cinviscmult * (2.0 * (vi[d] - f.velocity[d]));
    }
  }
  if (C1) {
    if (first) b_inversion(B, s.invb_det_thresh);
    b_renormalise(B, gradpt);
  }
  for (int d = 0; d < 3; ++d) {
    tpres[d] = tpres[d] + ALEt[d] + gradpt[d];
    tdiss[d] = tdiss[d] - VMon[d];
    tvisc[d] = tvisc[d] + VShear[d];
  }
}

// AddBoundaryContributions_to_ME2D.f90:96-402 (fixe/tapi, slip mode 1).
__device__ __forceinline__ void me_boundary2d(const SimDev& s, const DevBatch& b, int nb, int start, const double* vi, double roi,
                              double pressi, int lam, const double* grav, double* tpres, double* tdiss, double* tvisc) {
  const double pibmink = 10.0;
  double ro0 = s.den0, distpimin = s.dx;
  double VMon[2] = {0, 0}, VShear[2] = {0, 0}, RG_sum[2] = {0, 0}, ALEt[2] = {0, 0};
  const double g2[2] = {grav[0], grav[2]};
  const double v2[2] = {vi[0], vi[2]};
  for (int u = 0; u < nb; ++u) {
    const BdtEntry& e = b.P.bdt[start + u];
    const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
    double xpi = e.loc[0], ypi = e.loc[1];
    double IntWdS = e.bi[0], IntWdV = e.bi[2], IntWd1s0 = e.bi[5], IntWd3s0 = e.bi[6];
    double GravN = 0.0;
    for (int i = 0; i < 2; ++i) GravN = GravN + g2[i] * S.nnn[i];
    double sidevel[2] = {0.0, 0.0};
    if (S.zone_type == SPH_ZONE_TAPI) {
      sidevel[0] = S.velocity[0];
      sidevel[1] = S.velocity[2];
    }
    double Dvel0 = 2.0 * (v2[0] - sidevel[0]), Dvel1 = 2.0 * (v2[1] - sidevel[1]);
    double DvelN = Dvel0 * S.nnn[0] + Dvel1 * S.nnn[1];
    double distpi = fmax(ypi, distpimin);
    double pressib = pressi;
    double pressibmin = pibmink * ro0 * distpimin;
    if (DvelN <= 0.0 && pressib < pressibmin) pressib = pressibmin;
    double PressB = pressib - ro0 * GravN * distpi;
    double QiiIntWdS = IntWdS * (pressib + PressB) / roi;
    for (int i = 0; i < 2; ++i) {
      double RG = 0.0;
      for (int j = 0; j < 2; ++j) RG = RG + S.RN[i][j] * g2[j];
      RG = RG * IntWdV;
      RG_sum[i] = RG_sum[i] + RG;
    }
    ALEt[0] = ALEt[0] - S.nnn[0] * QiiIntWdS;
    ALEt[1] = ALEt[1] - S.nnn[1] * QiiIntWdS;
    if (xpi >= 0.0 && xpi <= S.length) {
      double Monvisc = s.alfa_mon * s.celerita * s.h;
      double TN = Monvisc * DvelN * IntWd3s0;
      double SVforce;
      if (lam == 1 || !S.laminar_no_slip_check) SVforce = 2.0 * s.kin_visc * S.slip * IntWd1s0;
      else SVforce = 0.0;
      for (int i = 0; i < 2; ++i) {
        VMon[i] = VMon[i] + TN * S.nnn[i];
        VShear[i] = VShear[i] + (2.0 * v2[i]) * SVforce;
      }
    }
  }
  const int acix[2] = {0, 2};
  for (int i = 0; i < 2; ++i) {
    tpres[acix[i]] = tpres[acix[i]] - RG_sum[i] - ALEt[i];
    tdiss[acix[i]] = tdiss[acix[i]] - VMon[i];
    tvisc[acix[i]] = tvisc[acix[i]] - VShear[i];
  }
}

// AddElasticBoundaryReaction_3D.f90:67-154 / _2D.f90:63-97; xi is
// pg%coord, vi pg%var (= pg%vel).
template <int DIM>
__device__ __forceinline__ void elastic_reaction(const SimDev& s, const DevBatch& b, int nb, int start, const double* xi,
                                                 const double* vi, double* R) {
  R[0] = R[1] = R[2] = 0.0;
  double zimin = 0.25 * s.dx;
  double celer02 = s.eps / s.den0;
  for (int u = 0; u < nb; ++u) {
    const BdtEntry& e = b.P.bdt[start + u];
    if (DIM == 3) {
      const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
      double zi = e.loc[2];
      if (zi < zimin && point_internal(f, e.loc[0], e.loc[1])) {
        double vin = 0.0;
        for (int sd = 0; sd < 3; ++sd) vin = vin + vi[sd] * f.T[sd][2];
        if (vin < 0.0) {
          double normreact = -(1.0 * celer02 * log((s.h + zi - zimin) / s.h) / s.h);
          for (int d = 0; d < 3; ++d) R[d] = R[d] + normreact * f.T[d][2];
        }
      }
    } else {
      const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
      double xpi = e.loc[0], ypi = e.loc[1];
      if (ypi < zimin && xpi > 0.0 && xpi < S.length) {
        double vin = 0.0;
        vin = vin + vi[0] * S.nnn[0];
        vin = vin + vi[1] * 0.0;
        vin = vin + vi[2] * S.nnn[1];
        if (vin < 0.0) {
          double normreact = -(1.0 * celer02 * log((s.h + ypi - zimin) / s.h) / s.h);
          R[0] = R[0] + normreact * S.nnn[0];
          R[2] = R[2] + normreact * S.nnn[1];
        }
      }
    }
  }
  if (DIM == 3 && s.nedges > 0) {
    // Reaction from close convex edges (AddElasticBoundaryReaction_3D.f90:106-153).
    // ReaFace(icbf) -- the face term above applied its test to the entry --
    // is recomputed from the entry here.  An edge counts only when both of
    // its faces are close faces of the particle without a face reaction;
    // the reference leaves the routine at the first edge that fails this,
    // and so does this loop.
    auto rea_face = [&](const BdtEntry& e) {
      const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
      return e.loc[2] < zimin && point_internal(f, e.loc[0], e.loc[1]);
    };
    for (int ne = 0; ne < s.nedges; ++ne) {
      const EdgeDev& E = b.edges[s.edge_off + ne];
      int nclose = 0;
      for (int u = 0; u < nb; ++u) {
        const BdtEntry& e = b.P.bdt[start + u];
        if ((e.clobonum == E.face[0] || e.clobonum == E.face[1]) && !rea_face(e)) nclose++;
      }
      if (nclose != 2) break;
      double scaprod = 0.0;
      for (int sd = 0; sd < 3; ++sd) scaprod = scaprod + (xi[sd] - E.gx[sd]) * E.comp[sd];
      const double edgelen2 = E.length * E.length;
      const double tau = scaprod / edgelen2;
      if (tau >= 0.0 && tau <= 1.0) {
        double QP[3], edgedist2 = 0.0;
        for (int sd = 0; sd < 3; ++sd) QP[sd] = xi[sd] - (E.gx[sd] + E.comp[sd] * tau);
        for (int sd = 0; sd < 3; ++sd) edgedist2 = edgedist2 + QP[sd] * QP[sd];
        const double zi = sqrt(edgedist2);
        if (zi < zimin) {
          double cosdir[3], vin = 0.0;
          for (int sd = 0; sd < 3; ++sd) cosdir[sd] = QP[sd] / zi;
          for (int sd = 0; sd < 3; ++sd) vin = vin + vi[sd] * cosdir[sd];
          if (vin < 0.0) {
            const double normreact = -(1.0 * celer02 * log(zi / zimin) / zimin);
            for (int sd = 0; sd < 3; ++sd) R[sd] = R[sd] + normreact * cosdir[sd];
          }
        }
      }
    }
  }
}

// ==========================================================================
// Neighbour lists (the replacement of
// CalcVarLength.f90:133-269).  One pass after the sort stores, per particle,
// the slots of its accepted neighbours (the particle itself excluded, its
// acceptance still counted for the NMAXPARTJ cap) in the reference's
// visiting order: runs in (y, x) order, slots increasing inside a run.  Only
// 4-byte slot indices are kept, never kernel values or separations (the
// reference keeps 60 B per slot); every pass recomputes those.  The list of a
// step serves its continuity pass and the next step's momentum pass, which
// see the same positions.
//
// Layout: entry k of particle p at ((p / 32) * cap + k) * 32 + p % 32, so a
// warp reads one 128-byte line per k.  An entry is slot | (run << 28); the
// run gives the FP32 form the cell-origin difference of the pair.
//
// The scan is warp-cooperative: the lanes of a warp that share a (y, x) cell
// column (nearly always all of them, particles being sorted z-fastest) stage
// the union of their 3-cell runs through shared memory 32 candidates at a
// time and test them in lockstep; each lane keeps the candidates of its own
// k-1..k+1 window, so its accepted sequence is exactly its reference order.
// ==========================================================================
constexpr int kSlotBits = 28;
constexpr int kSlotMask = (1 << kSlotBits) - 1;

// Entries are stored as 16-byte chunks of 4: chunk c of particle p sits at
// int4 index ((p / 32) * cap4 + c) * 32 + p % 32, so a warp reading chunk c
// of its 32 particles reads 512 contiguous bytes.
__device__ __forceinline__ size_t list_base4(int p, int cap4) {
  return (size_t)(p >> 5) * (size_t)cap4 * 32 + (size_t)(p & 31);
}


// A warp's list region -- its chunks 0 .. ceil(nmax / 4) - 1, 512 B each
// and contiguous -- requested into L2 by one bulk prefetch from lane 0, so
// the chunk loads of the pair loop find it in L2 instead of waiting on HBM
// (the lists of a full-size step, 4 B per pair, do not stay in L2 between
// the pass that writes them and the passes that read them).  A hint only:
// 16-byte aligned address, a size in multiples of 16 bytes, no completion.
__device__ __forceinline__ void prefetch_list_l2(const int* nlist, int p, int cap4, int nmax) {
  if ((threadIdx.x & 31) != 0 || nmax <= 0) return;
  const int4* a = reinterpret_cast<const int4*>(nlist) + (size_t)(p >> 5) * (size_t)cap4 * 32;
  const unsigned bytes = (unsigned)((nmax + 3) >> 2) * 512u;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(bytes) : "memory");
}

// Sequential reader that loads chunk c + 1 while chunk c is consumed, so
// the list's HBM latency overlaps four pairs' work.
struct ListPrefetcher {
  const int4* base;
  int4 cur, nxt;
  int nchunks;
  __device__ __forceinline__ void init(const int* nlist, int p, int cap4, int cnt) {
    base = reinterpret_cast<const int4*>(nlist) + list_base4(p, cap4);
    nchunks = (cnt + 3) >> 2;
    nxt = nchunks > 0 ? __ldg(base) : make_int4(0, 0, 0, 0);
  }
  __device__ __forceinline__ int get(int k) {
    if ((k & 3) == 0) {
      cur = nxt;
      int c = (k >> 2) + 1;
      if (c < nchunks) nxt = __ldg(base + (size_t)c * 32);
    }
    int e = cur.x;
    cur.x = cur.y;
    cur.y = cur.z;
    cur.z = cur.w;
    return e;
  }
};

// r^2 <= (2h)^2 (CalcVarLength.f90:223-228) is decided on the FP32
// screening copies outside [rr_lo, rr_hi], a band the host derives from the
// copies' rounding bounds, and in FP64, exactly as the reference, inside it.
// A group of lanes whose z cells span at most kRebaseSpan stages candidate z
// values re-based on the group's lowest cell, (kj - kmin) dcd + f_j, so the
// z difference costs one subtraction; the band covers that form's rounding
// too.  Candidates are rejected on the FP32 value alone; the window test
// (the candidate's z cell within one of the lane's), the NMAXPARTJ cap and
// the acceptance run only for the few that pass.
constexpr int kRebaseSpan = 6;

// FP32 r^2 of the lane and staged candidate xj.  REBASE: staged z values
// are (kj - kmin) dcdf + f_j and zi the lane's own; otherwise the raw
// offsets f_j with the cell difference formed here.
template <int DIM, bool REBASE>
__device__ __forceinline__ float screen_rf(const float4& xj, float ax, float ay, float zi, float fz, int ck, float dz) {
  float d0 = ax - xj.x;
  float d1 = (DIM == 3) ? ay - xj.y : 0.f;
  float d2 = REBASE ? zi - xj.z : (((float)ck - xj.w) * dz + fz) - xj.z;
  return __fmaf_rn(d2, d2, __fmaf_rn(d1, d1, __fmul_rn(d0, d0)));
}

// Screens the staged tile of nt candidates for one lane, branch-free: bit u
// of hitm is set unless candidate u's FP32 r^2 exceeds rr_hi (a certain
// rejection), bit u of lom when it is below rr_lo (a certain acceptance of
// the distance test; the caller still masks the lane's own 3-cell window,
// which a candidate closer than 2h can lie outside where cells are narrower
// than 2h).  Hits are about one candidate in nine; the band cases (hit, not
// low) are left to the caller.  Entries past nt are staged far away and
// never hit, so the tile is screened in blocks of 8.
template <int DIM, bool REBASE>
__device__ __forceinline__ void screen_tile(const float4* wbuf, int nt, float ax, float ay, float zi, float fz, int ck,
                                            float dz, float rr_lo, float rr_hi, unsigned& hitm, unsigned& lom) {
  unsigned hm = 0u, lm = 0u;
  for (int u0 = 0; u0 < nt; u0 += 8) {
    unsigned h8 = 0u, l8 = 0u;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      float rf = screen_rf<DIM, REBASE>(wbuf[u0 + c], ax, ay, zi, fz, ck, dz);
      if (!(rf > rr_hi)) h8 |= 1u << c;
      if (rf < rr_lo) l8 |= 1u << c;
    }
    hm |= h8 << u0;
    lm |= l8 << u0;
  }
  hitm = hm;
  lom = lm;
}

// screen_tile<DIM, true> on Blackwell's paired FP32 instructions: the tile
// is staged a second time as negated x, y, z arrays, and candidates u, u+1
// share each add, multiply and fused multiply-add (__fadd2_rn, __fmul2_rn,
// __ffma2_rn round each half as the scalar instruction does, x + (-y)
// rounds as x - y and fma(r, -1, y) as y - r, so every r^2 and both masks
// are bit-identical to screen_tile's).
template <int DIM>
__device__ __forceinline__ void screen_tile_x2(const float* nx, const float* ny, const float* nz, int nt, float ax,
                                               float ay, float zi, float rr_lo, float rr_hi, unsigned& hitm,
                                               unsigned& lom) {
  const float2 ax2 = make_float2(ax, ax), ay2 = make_float2(ay, ay), zi2 = make_float2(zi, zi);
  const float2 hi2 = make_float2(rr_hi, rr_hi), nlo2 = make_float2(-rr_lo, -rr_lo), m1 = make_float2(-1.f, -1.f);
  unsigned hm = 0u, lm = 0u;
#pragma unroll
  for (int u0 = 0; u0 < 32; u0 += 8) {
    if (u0 >= nt) break;
    unsigned h8 = 0u, l8 = 0u;
#pragma unroll
    for (int c = 4; c >= 0; c -= 4) {
      const float4 X = *reinterpret_cast<const float4*>(nx + u0 + c);
      const float4 Z = *reinterpret_cast<const float4*>(nz + u0 + c);
      float2 ra = __fadd2_rn(ax2, make_float2(X.x, X.y));
      float2 rb = __fadd2_rn(ax2, make_float2(X.z, X.w));
      const float2 za = __fadd2_rn(zi2, make_float2(Z.x, Z.y));
      const float2 zb = __fadd2_rn(zi2, make_float2(Z.z, Z.w));
      ra = __fmul2_rn(ra, ra);
      rb = __fmul2_rn(rb, rb);
      if (DIM == 3) {
        const float4 Y = *reinterpret_cast<const float4*>(ny + u0 + c);
        const float2 ya = __fadd2_rn(ay2, make_float2(Y.x, Y.y));
        const float2 yb = __fadd2_rn(ay2, make_float2(Y.z, Y.w));
        ra = __ffma2_rn(ya, ya, ra);
        rb = __ffma2_rn(yb, yb, rb);
      }
      ra = __ffma2_rn(za, za, ra);
      rb = __ffma2_rn(zb, zb, rb);
      // sign bits: rr_hi - r^2 < 0 exactly when r^2 > rr_hi, r^2 - rr_lo < 0
      // exactly when r^2 < rr_lo (finite inputs; a difference of two floats
      // is zero only when they are equal); one funnel shift per candidate
      // and mask moves the sign in, candidate u ending in bit u
      const float2 ha = __ffma2_rn(ra, m1, hi2), hb = __ffma2_rn(rb, m1, hi2);
      const float2 la = __fadd2_rn(ra, nlo2), lb = __fadd2_rn(rb, nlo2);
      h8 = __funnelshift_l(__float_as_uint(hb.y), h8, 1);
      h8 = __funnelshift_l(__float_as_uint(hb.x), h8, 1);
      h8 = __funnelshift_l(__float_as_uint(ha.y), h8, 1);
      h8 = __funnelshift_l(__float_as_uint(ha.x), h8, 1);
      l8 = __funnelshift_l(__float_as_uint(lb.y), l8, 1);
      l8 = __funnelshift_l(__float_as_uint(lb.x), l8, 1);
      l8 = __funnelshift_l(__float_as_uint(la.y), l8, 1);
      l8 = __funnelshift_l(__float_as_uint(la.x), l8, 1);
    }
    hm |= (~h8 & 0xffu) << u0;   // h8: rejected; l8: below rr_lo
    lm |= (l8 & 0xffu) << u0;
  }
  hitm = hm;
  lom = lm;
}

// Whether any staged candidate u0 <= u < nt lies in the lane's 3-cell z
// window (the truncation test once NMAXPARTJ is reached; rare).
__device__ __forceinline__ bool in_window(float kj, int ck) { return fabsf(kj - (float)ck) <= 1.0f; }

// Bits u of a 32-candidate tile with lo <= u < hi (lo, hi relative to the
// tile's first slot, any sign).
__device__ __forceinline__ unsigned window_mask(int lo, int hi) {
  lo = lo < 0 ? 0 : lo;
  hi = hi > 32 ? 32 : hi;
  if (hi <= lo) return 0u;
  const unsigned upto = hi == 32 ? 0xffffffffu : (1u << hi) - 1u;
  return upto & ~((1u << lo) - 1u);
}

__device__ __forceinline__ bool window_candidate(const float4* wbuf, int u0, int nt, int ck) {
  for (int u = u0; u < nt; ++u)
    if (in_window(wbuf[u].w, ck)) return true;
  return false;
}

template <int DIM>
__global__ void __launch_bounds__(kBlock, 4) k_neighbour_lists(DevBatch b) {
  __shared__ SimDev s;
  __shared__ float4 cbuf[kBlock];
  __shared__ __align__(16) float cneg[3][kBlock];   // the tile again: -x, -y, -z (paired screening)
  int cur = -1;
  const Particles& P = b.P;
  const int lane = threadIdx.x & 31;
  float4* wbuf = cbuf + (threadIdx.x & ~31);
  float* wnx = &cneg[0][threadIdx.x & ~31];
  float* wny = &cneg[1][threadIdx.x & ~31];
  float* wnz = &cneg[2][threadIdx.x & ~31];
  constexpr int NR = (DIM == 3) ? 9 : 3;
  const unsigned FULL = 0xffffffffu;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen;
    double4 xd = make_double4(0.0, 0.0, 0.0, 0.0);
    float4 xf = make_float4(0.f, 0.f, 0.f, 0.f);
    int ci = 0, cj = 0, ck = 0;
    bool on = false;
    if (active) {
      xd = P.X[p];
      xf = P.XF[p];
      on = particle_cell(s, xd.x, xd.y, xd.z, ci, cj, ck);
      if (!on) set_status(dyn, SPH_ERR_INVALID_ARGUMENT);   // state not re-sorted after a move
    }
    int colkey = on ? (cj * s.ncd[0] + ci) : -1;
    unsigned remaining = __ballot_sync(FULL, on);
    int cnt = 0, nacc = 0, cand = 0;
    bool trunc = false;
    const int cap = s.nmaxpartj;
    int4* out = reinterpret_cast<int4*>(b.nlist) + list_base4(p, b.list_cap4);
    int4 pend = make_int4(0, 0, 0, 0);   // entries not yet written, oldest in x
    const float rr_lo = s.rr_lo, rr_hi = s.rr_hi, dz = s.dcdf[2];
    bool full = cap <= 0;                            // NMAXPARTJ reached
    while (remaining) {
      int leader = __ffs(remaining) - 1;
      int key = __shfl_sync(FULL, colkey, leader);
      unsigned group = __ballot_sync(FULL, on && colkey == key) & remaining;
      remaining &= ~group;
      bool mine = (group >> lane) & 1u;
      int kmin = __reduce_min_sync(FULL, mine ? ck : 0x7fffffff);
      int kmax = __reduce_max_sync(FULL, mine ? ck : -0x7fffffff);
      int gci = __shfl_sync(FULL, ci, leader);
      int gcj = __shfl_sync(FULL, cj, leader);
      const bool rebase = kmax - kmin <= kRebaseSpan;          // uniform over the warp
      const float zi = rebase ? (float)(ck - kmin) * dz + xf.z : 0.f;
      for (int r = 0; r < NR; ++r) {
        int jr = (DIM == 3) ? gcj - 1 + r / 3 : gcj;
        int ir = gci - 1 + ((DIM == 3) ? r % 3 : r);
        if (ir < 1 || ir > s.ncd[0] || jr < 1 || jr > s.ncd[1]) continue;
        int klo = kmin > 1 ? kmin - 1 : 1;
        int khi = kmax < s.ncd[2] ? kmax + 1 : s.ncd[2];
        int base = s.cell_off + ((jr - 1) * s.ncd[0] + (ir - 1)) * s.ncd[2];
        int ub = __ldg(P.cell_start + base + klo - 1);
        int ue = __ldg(P.cell_start + base + khi);
        // this lane's own window in the run, cells ck-1..ck+1: the slots the
        // reference visits (CalcVarLength.f90's 27-cell block)
        int wlo = 0, whi = 0;
        if (mine) {
          int ml = ck > 1 ? ck - 1 : 1, mh = ck < s.ncd[2] ? ck + 1 : s.ncd[2];
          wlo = __ldg(P.cell_start + base + ml - 1);
          whi = __ldg(P.cell_start + base + mh);
          cand += whi - wlo;
        }
        float Dx = (float)(gci - ir) * s.dcdf[0];
        float Dy = (DIM == 3) ? (float)(gcj - jr) * s.dcdf[1] : 0.f;
        float ax = Dx + xf.x, ay = Dy + xf.y;
        const int tag = r << kSlotBits;
        for (int c0 = ub; c0 < ue; c0 += 32) {
          int cidx = c0 + lane;
          float4 st = (cidx < ue) ? P.XF[cidx] : make_float4(3.0e18f, 3.0e18f, 3.0e18f, -1.0e9f);
          if (rebase && cidx < ue) st.z = (st.w - (float)kmin) * dz + st.z;
          __syncwarp();
          wbuf[lane] = st;
          if (rebase) {
            wnx[lane] = -st.x;
            wny[lane] = -st.y;
            wnz[lane] = -st.z;
          }
          __syncwarp();
          if (!mine) continue;
          int nt = ue - c0 < 32 ? ue - c0 : 32;
          // phase 1: screening masks of the tile
          unsigned hitm, lom;
          if (rebase) screen_tile_x2<DIM>(wnx, wny, wnz, nt, ax, ay, zi, rr_lo, rr_hi, hitm, lom);
          else screen_tile<DIM, false>(wbuf, nt, ax, ay, zi, xf.z, ck, dz, rr_lo, rr_hi, hitm, lom);
          if (full) {
            // NMAXPARTJ reached: every later candidate of the window is refused
            if (!trunc && window_candidate(wbuf, 0, nt, ck)) trunc = true;
            continue;
          }
          // only the lane's own window counts: the warp's union of runs
          // reaches two z cells away from some lanes, and where the cells are
          // narrower than 2h (CreaGrid rounds the cell count to nearest) a
          // candidate there can lie within 2h without being the reference's
          // neighbour; with cells at least 2h wide such a candidate is never
          // a hit below the band, and band hits are tested below
          if (s.narrow_z) hitm &= window_mask(wlo - c0, whi - c0);
          // phase 2a (rare): resolve band hits -- outside the lane's window
          // (the reference never visits those) or failing the FP64 test
          // they are dropped; hitm then holds exactly the accepted ones
          unsigned band = hitm & ~lom;
          while (band) {
            int u = __ffs(band) - 1;
            band &= band - 1;
            bool keep = in_window(wbuf[u].w, ck);
            if (keep) {
              double4 xq = P.X[c0 + u], xi = P.X[p];
              double r0 = xi.x - xq.x, r1 = xi.y - xq.y, r2 = xi.z - xq.z;
              double rr = r0 * r0 + r1 * r1 + r2 * r2;
              keep = !(rr > s.square_doubleh);
            }
            if (!keep) hitm &= ~(1u << u);
          }
          if (nacc + __popc(hitm) >= cap) {
            // reaching NMAXPARTJ in this tile (rare): accepted ones in
            // visiting order up to the cap, then the truncation test
            while (hitm) {
              int u = __ffs(hitm) - 1;
              hitm &= hitm - 1;
              nacc++;
              int q = c0 + u;
              if (q != p) {
                pend.x = pend.y;
                pend.y = pend.z;
                pend.z = pend.w;
                pend.w = q | tag;
                cnt++;
                if ((cnt & 3) == 0) out[(size_t)((cnt >> 2) - 1) * 32] = pend;
              }
              if (nacc >= cap) {
                full = true;
                if (window_candidate(wbuf, u + 1, nt, ck)) trunc = true;   // window candidates follow
                break;
              }
            }
            continue;
          }
          // phase 2b: append the accepted ones in visiting order (the lane
          // itself counted, not stored)
          nacc += __popc(hitm);
          unsigned self = (unsigned)(p - c0) < (unsigned)nt ? 1u << (p - c0) : 0u;
          hitm &= ~self;
          const int qbase = c0 | tag;                 // c0 + u < 2^28: no carry into the run bits
          while (hitm) {
            int u = __ffs(hitm) - 1;
            hitm &= hitm - 1;
            pend.x = pend.y;
            pend.y = pend.z;
            pend.z = pend.w;
            pend.w = qbase + u;
            cnt++;
            if ((cnt & 3) == 0) out[(size_t)((cnt >> 2) - 1) * 32] = pend;
          }
        }
      }
    }
    if (cnt & 3) {
      // flush the last partial chunk, entries moved to its front
      int rem = cnt & 3;
      int4 w = pend;
      if (rem == 1) w = make_int4(pend.w, 0, 0, 0);
      else if (rem == 2) w = make_int4(pend.z, pend.w, 0, 0);
      else w = make_int4(pend.y, pend.z, pend.w, 0);
      out[(size_t)(cnt >> 2) * 32] = w;
    }
    if (active) {
      b.ncount[p] = cnt;
      if (trunc) atomicOr(&dyn->warnings, SPH_WARN_NEIGHBOURS_TRUNCATED);
    }
    block_count2(b.counters, cand, nacc);
    int m = warp_max(nacc);
    if (lane == 0 && m > 0) atomicMax(&dyn->max_neigh, m);
  }
}

// ==========================================================================
// Momentum, FP64 form: RHS_momentum_equation + inter_EqMoto + viscomon +
// viscomorris + AddBoundaryContributions_to_ME3D/2D +
// AddElasticBoundaryReaction_3D/2D, optionally fused with Leapfrog_momentum,
// velocity_smoothing_2 (TetaV = 0), Leapfrog_trajectories and the CFL part of
// time_step_duration.  The list is drained in warp lockstep.
// ==========================================================================
// CalcVarLength.f90:285-324 (3D, C1_BE): the fluid part of the
// renormalisation matrices, summed over the particle's list in its order.
// A pair adds (x_j - x_i)_c grad_W_k m_j / rho_j to B(k,c), grad_W that of
// the anti-cluster kernel for B_ren_gradp and of the beta-spline for
// B_ren_divu (grad_W_sub.f90:52-91, 3D); a pair with r >= 2h adds nothing
// (CalcVarLength.f90:254), nor does a zero gradient (r < 1e-6 h, the
// particle itself): the sums start at +0, so skipping a +-0 addend leaves
// them as they are.  The frontier terms are added by the momentum (first
// step) and continuity passes, which also invert.  One sqrt and the
// division r / h are shared by the range test and both gradients; the
// constant factors come from the host (SimDev::c1_w*).  The pair's twelve
// divisions by |r| and rho_j go through one correctly rounded reciprocal
// of each (div_rn: the IEEE quotients, bit for bit).
// The 2D SA-SPH frontier terms of the renormalisation matrices, -RN IntWdV
// per close side (AddBoundaryContribution_to_CE2D.f90:81-94 for both
// matrices in every continuity pass; AddBoundaryContributions_to_ME2D.f90:
// 290-300 for B_ren_gradp on the first step, GRADP_ONLY), then their
// inversion (SASPH_continuity.f90:112-119, ME2D.f90:377-383).  In 2D the
// matrices have a zero y row and column, so their determinant is zero and
// the inversion always gives the -I of B_ren_gradp_inversion.f90:67-72
// (a positive invb_det_thresh is required); renormalising with -I leaves
// every vector as it is, so the rates are the plain form's and only the
// matrices themselves are formed here.
template <bool GRADP_ONLY>
__global__ void k_c1_frontier_2d(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  const int total = P.total_slots;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    const SimDyn* dyn = b.dyn + tl.sim;
    if (!s.c1_be || dyn->frozen || (GRADP_ONLY && dyn->step != 0)) continue;
    const int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + dyn->nag) continue;
    const bool divu = !GRADP_ONLY && s.c1_divu;
    double Bg[9], Bd[9];
    load_b(P.BG, total, p, Bg);
    if (divu) load_b(P.BD, total, p, Bd);
    const int nb = P.bdt_count[p];
    const int start = nb > 0 ? P.bdt_start[p] : 0;
    for (int u = 0; u < nb; ++u) {
      const BdtEntry& e = P.bdt[start + u];
      const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
      const double IntWdV = e.bi[2];
      const int ax[2] = {0, 2};
      for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 2; ++c) {
          const double aux = -S.RN[a][c] * IntWdV;
          Bg[3 * ax[a] + ax[c]] = Bg[3 * ax[a] + ax[c]] + aux;
          if (divu) Bd[3 * ax[a] + ax[c]] = Bd[3 * ax[a] + ax[c]] + aux;
        }
    }
    if (divu) {
      b_inversion(Bd, s.invb_det_thresh);
      store_b(P.BD, total, p, Bd);
    }
    b_inversion(Bg, s.invb_det_thresh);
    store_b(P.BG, total, p, Bg);
  }
}

// 2D (DIM = 2): grad_W_sub.f90:79-88 scales both gradients by h 10/7
// (beta-spline) and h 4/3 (anti-cluster); y is zero throughout.
template <int DIM>
__global__ void __launch_bounds__(kBlock, 2) k_renormalisation(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  const int total = P.total_slots;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (!s.c1_be) continue;
    const bool divu = s.c1_divu != 0;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + b.dyn[tl.sim].nag;
    double4 xi = make_double4(0.0, 0.0, 0.0, 0.0);
    int cnt = 0;
    if (active) {
      xi = P.X[p];
      cnt = b.ncount[p];
    }
    double Bg[9], Bd[9];
    for (int k = 0; k < 9; ++k) Bg[k] = Bd[k] = 0.0;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    for (int k = 0; k < nmax; ++k) {
      int e = lr.get(k);
      if (k >= cnt) continue;
      int q = e & kSlotMask;
      double4 xj = P.X[q];
      double r[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
      double abs_r = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      double qh = div_rn(abs_r, s.h, s.rcp_h);
      if ((int)qh >= 2 || abs_r < s.h * 1.0e-6) continue;
      const double mj = xj.w, rhoj = P.RP[q].x;
      const double w = 2.0 - qh;
      double go[3];
      // anti-cluster kernel (q <= 2 here)
      const double rcp_r = __drcp_rn(abs_r), rcp_rhoj = __drcp_rn(rhoj);
      double t = div_rn(-(3.0 * (w * w) * s.c1_w2), s.h, s.rcp_h);
      for (int c = 0; c < 3; ++c) {
        double gw = div_rn(t * r[c], abs_r, rcp_r);
        if (DIM == 2) gw = gw * s.h * 4.0 / 3.0;
        go[c] = div_rn(gw * mj, rhoj, rcp_rhoj);
      }
      for (int c = 0; c < 3; ++c)
        for (int kk = 0; kk < 3; ++kk) Bg[3 * kk + c] = Bg[3 * kk + c] + r[c] * go[kk];
      if (divu) {
        // beta-spline (q < 2 here)
        t = div_rn(qh <= 1.0 ? s.c1_w1a * (9.0 / 4.0 * (qh * qh) - 3.0 * qh) : -(s.c1_w1b * (w * w)), s.h, s.rcp_h);
        for (int c = 0; c < 3; ++c) {
          double gw = div_rn(t * r[c], abs_r, rcp_r);
          if (DIM == 2) gw = gw * s.h * 10.0 / 7.0;
          go[c] = div_rn(gw * mj, rhoj, rcp_rhoj);
        }
        for (int c = 0; c < 3; ++c)
          for (int kk = 0; kk < 3; ++kk) Bd[3 * kk + c] = Bd[3 * kk + c] + r[c] * go[kk];
      }
    }
    if (active) {
      store_b(P.BG, total, p, Bg);
      if (divu) store_b(P.BD, total, p, Bd);
    }
  }
}

// C1: with input_any_t%C1_BE the pressure terms are renormalised with
// B_ren_gradp (3D only).
// BATCH (not with C1): two list entries' records are requested before the
// first one's arithmetic, so the second pair's gathers wait behind the
// first pair's FP64 divisions instead of after them; the terms are formed
// and summed in the same order, so the results are the same bits.
template <int DIM, bool FUSED, bool C1 = false, bool BATCH = false>
__global__ void __launch_bounds__(kBlock, 2) k_momentum(DevBatch b) {
  __shared__ SimDev s;
  __shared__ double stpres[3][kBlock];   // the wall pressure term, kept out of the pair loop's registers
  int cur = -1;
  const Particles& P = b.P;
  const double GI = (double)9.80665f;   // Static_allocation_module.f90:72, a default-REAL literal
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    const double* geff = dyn->geff;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag;
    if (FUSED && active && dyn->frozen) {
      // a finished simulation of a batch: carry the record through the sort
      double4 v4 = P.V[p];
      double2 rp = P.RP[p];
      P.X2[p] = P.X[p];
      P.V2[p] = make_double4(v4.x, v4.y, v4.z, rp.x);
      P.P2[p] = rp.y;
      P.I2[p] = P.I[p];
      P.L2[p] = P.L[p];
      active = false;
    }
    double4 xi = make_double4(0.0, 0.0, 0.0, 0.0);
    double vi[3] = {0.0, 0.0, 0.0};
    double rhoi = 1.0, pi = 0.0;
    int cnt = 0;
    double tdiss[3] = {0, 0, 0}, tvisc[3] = {0, 0, 0};
    if (active) {
      xi = P.X[p];
      double4 v4 = P.V[p];
      double2 rp = P.RP[p];
      vi[0] = v4.x;
      vi[1] = v4.y;
      vi[2] = v4.z;
      rhoi = rp.x;
      pi = rp.y;
      cnt = b.ncount[p];
      const int nb = P.bdt_count[p];
      double tpres[3] = {0, 0, 0};
      // C1: on the first step the frontiers complete B_ren_gradp and it is
      // inverted, for every particle (RHS_momentum_equation.f90:130-150)
      const bool c1 = C1 && s.c1_be;
      const bool first = c1 && dyn->step == 0;
      if (c1) {
        double B[9];
        load_b(P.BG, P.total_slots, p, B);
        if (nb > 0)
          me_boundary3d<true>(s, b, nb, P.bdt_start[p], vi, rhoi, pi, P.L[p], geff, tpres, tdiss, tvisc, B, first);
        else if (first)
          b_inversion(B, s.invb_det_thresh);
        if (first) store_b(P.BG, P.total_slots, p, B);
      } else if (nb > 0) {
        const int lam = P.L[p];
        const int bstart = P.bdt_start[p];
        if (DIM == 3) me_boundary3d(s, b, nb, bstart, vi, rhoi, pi, lam, geff, tpres, tdiss, tvisc);
        else me_boundary2d(s, b, nb, bstart, vi, rhoi, pi, lam, geff, tpres, tdiss, tvisc);
      }
      for (int d = 0; d < 3; ++d) stpres[d][threadIdx.x] = tpres[d];
    }
    double tp0 = 0, tp1 = 0, tp2 = 0, al0 = 0, al1 = 0, al2 = 0;
    double td0 = tdiss[0], td1 = tdiss[1], td2 = tdiss[2];
    double tv0 = tvisc[0], tv1 = tvisc[1], tv2 = tvisc[2];
    double rs0 = 0, rs1 = 0, rs2 = 0;
    const double celt = s.celerita + s.celerita;
    const double rcp_rhoi = __drcp_rn(rhoi);
    const bool morris = s.kin_visc > 1.0e-12;
    const double nu = s.kin_visc;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    auto pair = [&](const double4& xj, const double4& vj, const double2& rpj) {
      double r0 = xi.x - xj.x, r1 = xi.y - xj.y, r2 = xi.z - xj.z;
      double rr = r0 * r0 + r1 * r1 + r2 * r2;
      double PK1, PK2, PK3;
      kernel_values(s, rr, PK1, PK2, PK3);
      double rhoj = rpj.x, pj = rpj.y, amassj = xj.w;
      double dv0 = vj.x - vi[0], dv1 = vj.y - vi[1], dv2 = vj.z - vi[2];
      // pressure gradient and ALE1 terms, inter_EqMoto.f90:195-221
      // the two divisions by rho_i rho_j and the one by rho_i share correctly
      // rounded reciprocals (div_rn: the IEEE quotients, bit for bit)
      const double rr_ij = rhoi * rhoj, rcp_rr = __drcp_rn(rr_ij);
      double alpha = div_rn(pj - pi, rr_ij, rcp_rr);
      tp0 = tp0 + -(amassj * alpha * r0 * PK3);
      if (DIM == 3) tp1 = tp1 + -(amassj * alpha * r1 * PK3);
      tp2 = tp2 + -(amassj * alpha * r2 * PK3);
      double alpha2 = div_rn(pi * (div_rn(rhoj, rhoi, rcp_rhoi) + 1.0) + pj * (rhoi / rhoj - 1.0), rr_ij, rcp_rr);
      al0 = al0 - amassj * alpha2 * r0 * PK3;
      if (DIM == 3) al1 = al1 - amassj * alpha2 * r1 * PK3;
      al2 = al2 - amassj * alpha2 * r2 * PK3;
      // viscomon.f90:54-73
      double vrij = (DIM == 3) ? -(dv0 * r0) - dv1 * r1 - dv2 * r2 : -(dv0 * r0) - dv2 * r2;
      double TermMon = s.alfa_mon * celt * s.h / (rhoi + rhoj);
      double mtv = amassj * TermMon * vrij;
      td0 = td0 + (mtv * r0 * PK2 + 0.0);
      if (DIM == 3) td1 = td1 + (mtv * r1 * PK2 + 0.0);
      td2 = td2 + (mtv * r2 * PK2 + 0.0);
      // viscomorris.f90:60-71
      if (morris) {
        double rt = nu * rhoi + nu * rhoj + 1.0e-3;
        double anuitilde = 4.0 * (nu * nu);
        double factivis = amassj * anuitilde / rt;
        double w0 = factivis * (-(dv0 * PK2 * rr));
        double w2 = factivis * (-(dv2 * PK2 * rr));
        tv0 = tv0 + w0;
        rs0 = rs0 + w0;
        if (DIM == 3) {
          double w1 = factivis * (-(dv1 * PK2 * rr));
          tv1 = tv1 + w1;
          rs1 = rs1 + w1;
        }
        tv2 = tv2 + w2;
        rs2 = rs2 + w2;
      }
    };
    if (BATCH) {
      for (int k = 0; k < nmax; k += 2) {
        const int e0 = lr.get(k);
        const int e1 = k + 1 < nmax ? lr.get(k + 1) : 0;
        const bool u0 = k < cnt, u1 = k + 1 < cnt;
        double4 x0 = make_double4(0.0, 0.0, 0.0, 0.0), v0 = x0, x1 = x0, v1 = x0;
        double2 p0 = make_double2(0.0, 0.0), p1 = p0;
        if (u0) {
          const int q = e0 & kSlotMask;
          x0 = P.X[q]; v0 = P.V[q]; p0 = P.RP[q];
        }
        if (u1) {
          const int q = e1 & kSlotMask;
          x1 = P.X[q]; v1 = P.V[q]; p1 = P.RP[q];
        }
        if (u0) pair(x0, v0, p0);
        if (u1) pair(x1, v1, p1);
      }
    } else {
      for (int k = 0; k < nmax; ++k) {
        int e = lr.get(k);
        if (k >= cnt) continue;
        int q = e & kSlotMask;
        pair(P.X[q], P.V[q], P.RP[q]);
      }
    }
    double dtc = 1.0e300;
    if (active) {
      if (C1 && s.c1_be) {
        // inter_EqMoto.f90:255-260
        double B[9], tp[3] = {tp0, tp1, tp2};
        load_b(P.BG, P.total_slots, p, B);
        b_renormalise(B, tp);
        tp0 = tp[0];
        tp1 = tp[1];
        tp2 = tp[2];
      }
      double tpres[3];
      tpres[0] = stpres[0][threadIdx.x] + tp0 + al0;
      tpres[1] = stpres[1][threadIdx.x] + tp1 + al1;
      tpres[2] = stpres[2][threadIdx.x] + tp2 + al2;
      const int nb = P.bdt_count[p];
      const int bstart = nb > 0 ? P.bdt_start[p] : 0;
      // laminar_flag, inter_EqMoto.f90:269-283
      int lam_new = 0;
      if (s.kin_visc > 0.0) {
        double absv_pres = sqrt(tpres[0] * tpres[0] + tpres[1] * tpres[1] + tpres[2] * tpres[2]) + GI;
        double absv_morris = sqrt(rs0 * rs0 + rs1 * rs1 + rs2 * rs2);
        double weight = 0.0;
        if (absv_pres != 0.0) weight = absv_morris / absv_pres * 100.0;
        lam_new = (weight > 5.0 || absv_pres == 0.0) ? 1 : 0;
      }
      double acc[3];
      acc[0] = tpres[0] + td0 + tv0 + geff[0];
      acc[1] = tpres[1] + td1 + tv1 + geff[1];
      acc[2] = tpres[2] + td2 + tv2 + geff[2];
      if (nb > 0) {
        double R[3];
        const double xa[3] = {xi.x, xi.y, xi.z};
        elastic_reaction<DIM>(s, b, nb, bstart, xa, vi, R);
        for (int d = 0; d < 3; ++d) acc[d] = acc[d] + R[d];
      }
      if (FUSED) {
        double dtvel = dyn->dtvel, dt = dyn->dt;
        double vn[3], xn[3];
        for (int d = 0; d < 3; ++d) vn[d] = vi[d] + dtvel * acc[d];
        xn[0] = xi.x + dt * vn[0];
        xn[1] = xi.y + dt * vn[1];
        xn[2] = xi.z + dt * vn[2];
        P.X2[p] = make_double4(xn[0], xn[1], xn[2], xi.w);
        P.V2[p] = make_double4(vn[0], vn[1], vn[2], rhoi);
        P.P2[p] = pi;
        P.I2[p] = P.I[p];
        P.L2[p] = (uint8_t)lam_new;
        double U = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
        // with velocity smoothing the CFL minimum is taken on the smoothed
        // velocities (k_velocity_smoothing_apply), which also moves X2
        if (!(s.teta_v > 1.0e-9)) dtc = s.cfl * 2.0 * s.h / (s.celerita + U);
      } else {
        P.ACC[p] = make_double4(acc[0], acc[1], acc[2], 0.0);
        P.L[p] = (uint8_t)lam_new;
      }
    }
    if (FUSED) {
      double m = warp_min(dtc);
      if ((threadIdx.x & 31) == 0 && m < 1.0e300)
        atomicMin(&dyn->dtmin_bits, (unsigned long long)__double_as_longlong(m));
    }
  }
}

// SASPH_continuity.f90:89-169 with AddBoundaryContribution_to_CE3D/2D: the
// wall term of drho/dt, starting value of the continuity sum (FP64).
template <int DIM>
__device__ __forceinline__ double continuity_boundary(const SimDev& s, const DevBatch& b, SimDyn* dyn, int nb,
                                                      int bstart, const double4& vi, double rhoi) {
  const Particles& P = b.P;
  double gu0 = 0, gv1 = 0, gw2 = 0;
  if (DIM == 3) {
    double gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
    const double var[3] = {vi.x, vi.y, vi.z};
    for (int u = 0; u < nb; ++u) {
      const BdtEntry& e = P.bdt[bstart + u];
      const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
      if (!(e.loc[2] > 0.0)) continue;
      double dp = 0.0;
      for (int d = 0; d < 3; ++d) dp = dp + (2.0 * (f.velocity[d] - var[d])) * f.T[d][2];
      double dvel[3] = {dp * f.T[0][2], dp * f.T[1][2], dp * f.T[2][2]};
      double av[3];
      for (int i = 0; i < 3; ++i) {
        double a = 0.0;
        for (int k = 0; k < 3; ++k) a = a + f.T[i][k] * e.bi[3 + k];
        av[i] = a;
      }
      for (int d = 0; d < 3; ++d) {
        gu[d] = gu[d] - dvel[0] * av[d];
        gv[d] = gv[d] - dvel[1] * av[d];
        gw[d] = gw[d] - dvel[2] * av[d];
      }
    }
    gu0 = gu[0];
    gv1 = gv[1];
    gw2 = gw[2];
    atomicMax(&dyn->ncbf_max, nb);
  } else {
    const double var2[2] = {vi.x, vi.z};
    double gu_x = 0.0, gw_z = 0.0;
    for (int u = 0; u < nb; ++u) {
      const BdtEntry& e = P.bdt[bstart + u];
      const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
      double IntWdS = e.bi[0];
      double dvel0, dvel1;
      if (S.zone_type == SPH_ZONE_TAPI) {
        dvel0 = 2.0 * (S.velocity[0] - var2[0]);
        dvel1 = 2.0 * (S.velocity[2] - var2[1]);
      } else {
        dvel0 = 2.0 * (-var2[0]);
        dvel1 = 2.0 * (-var2[1]);
      }
      gu_x = gu_x - dvel0 * S.nnn[0] * IntWdS;
      gw_z = gw_z - dvel1 * S.nnn[1] * IntWdS;
    }
    gu0 = gu_x;
    gw2 = gw_z;
  }
  return 0.0 - rhoi * (gu0 + gv1 + gw2);
}

// SASPH_continuity.f90:89-169 with C1_BE (3D): the frontiers complete the
// renormalisation matrices (AddBoundaryContribution_to_CE3D.f90:93-112),
// both are inverted for every particle, and with C1_divu the wall velocity
// gradients are renormalised before they enter drho/dt.
__device__ __forceinline__ double continuity_boundary_c1(const SimDev& s, const DevBatch& b, SimDyn* dyn, int nb,
                                                         int bstart, const double4& vi, double rhoi, int p) {
  const Particles& P = b.P;
  const int total = P.total_slots;
  const bool divu = s.c1_divu != 0;
  double Bg[9], Bd[9];
  load_b(P.BG, total, p, Bg);
  if (divu) load_b(P.BD, total, p, Bd);
  double gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
  const double var[3] = {vi.x, vi.y, vi.z};
  for (int u = 0; u < nb; ++u) {
    const BdtEntry& e = P.bdt[bstart + u];
    const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
    if (!(e.loc[2] > 0.0)) continue;
    if (divu) add_frontier_b(f, e, Bd);
    add_frontier_b(f, e, Bg);
    double dp = 0.0;
    for (int d = 0; d < 3; ++d) dp = dp + (2.0 * (f.velocity[d] - var[d])) * f.T[d][2];
    double dvel[3] = {dp * f.T[0][2], dp * f.T[1][2], dp * f.T[2][2]};
    double av[3];
    for (int i = 0; i < 3; ++i) {
      double a = 0.0;
      for (int k = 0; k < 3; ++k) a = a + f.T[i][k] * e.bi[3 + k];
      av[i] = a;
    }
    for (int d = 0; d < 3; ++d) {
      gu[d] = gu[d] - dvel[0] * av[d];
      gv[d] = gv[d] - dvel[1] * av[d];
      gw[d] = gw[d] - dvel[2] * av[d];
    }
  }
  if (divu) b_inversion(Bd, s.invb_det_thresh);
  b_inversion(Bg, s.invb_det_thresh);
  store_b(P.BG, total, p, Bg);
  if (divu) store_b(P.BD, total, p, Bd);
  if (nb == 0) return 0.0;
  atomicMax(&dyn->ncbf_max, nb);
  if (divu) {
    b_renormalise(Bd, gu);
    b_renormalise(Bd, gv);
    b_renormalise(Bd, gw);
  }
  return 0.0 - rhoi * (gu[0] + gv[1] + gw[2]);
}

// Continuity, FP64 form: SASPH_continuity + Continuity_Equation, optionally
// fused with Leapfrog_continuity and the EoS.  C1 (3D): the renormalised
// form, Continuity_Equation.f90:119-126,201-217 -- the whole velocity
// gradient vectors are summed, and renormalised with B_ren_divu when
// C1_divu is set; their trace equals the plain form's sum bit for bit.
// BATCH (not with C1): two list entries' records requested before the
// first one's arithmetic, as in k_momentum; the same sums.
template <int DIM, bool FUSED, bool C1 = false, bool BATCH = false>
__global__ void __launch_bounds__(kBlock, 2) k_continuity(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !(FUSED && dyn->frozen);
    double4 xi = make_double4(0.0, 0.0, 0.0, 0.0);
    double4 vi = make_double4(0.0, 0.0, 0.0, 0.0);
    double rhoi = 1.0, dden = 0.0;
    int cnt = 0;
    if (active) {
      xi = P.X[p];
      vi = P.V[p];
      rhoi = P.RP[p].x;
      cnt = b.ncount[p];
      int nb = P.bdt_count[p];
      if (C1 && s.c1_be) dden = continuity_boundary_c1(s, b, dyn, nb, nb > 0 ? P.bdt_start[p] : 0, vi, rhoi, p);
      else if (nb > 0) dden = continuity_boundary<DIM>(s, b, dyn, nb, P.bdt_start[p], vi, rhoi);
    }
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    double g1[3] = {0, 0, 0}, g2[3] = {0, 0, 0}, g3[3] = {0, 0, 0};
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    auto pair = [&](const double4& xj, const double4& vj) {
      double r0 = xi.x - xj.x, r1 = xi.y - xj.y, r2 = xi.z - xj.z;
      double rr = r0 * r0 + r1 * r1 + r2 * r2;
      double PK1, PK2, PK3;
      kernel_values(s, rr, PK1, PK2, PK3);
      double c = rhoi * vj.w * PK1;     // rhoi * (amassj / rhoj) * PK1
      if (C1) {
        const double c0 = c * (vj.x - vi.x), c1 = c * (vj.y - vi.y), c2 = c * (vj.z - vi.z);
        g1[0] = g1[0] + c0 * r0;
        g1[1] = g1[1] + c0 * r1;
        g1[2] = g1[2] + c0 * r2;
        g2[0] = g2[0] + c1 * r0;
        g2[1] = g2[1] + c1 * r1;
        g2[2] = g2[2] + c1 * r2;
        g3[0] = g3[0] + c2 * r0;
        g3[1] = g3[1] + c2 * r1;
        g3[2] = g3[2] + c2 * r2;
      } else {
        a1 = a1 + c * (vj.x - vi.x) * r0;
        if (DIM == 3) a2 = a2 + c * (vj.y - vi.y) * r1;
        a3 = a3 + c * (vj.z - vi.z) * r2;
      }
    };
    if (BATCH) {
      for (int k = 0; k < nmax; k += 2) {
        const int e0 = lr.get(k);
        const int e1 = k + 1 < nmax ? lr.get(k + 1) : 0;
        const bool u0 = k < cnt, u1 = k + 1 < cnt;
        double4 x0 = make_double4(0.0, 0.0, 0.0, 0.0), v0 = x0, x1 = x0, v1 = x0;
        if (u0) {
          const int q = e0 & kSlotMask;
          x0 = P.X[q]; v0 = P.V[q];
        }
        if (u1) {
          const int q = e1 & kSlotMask;
          x1 = P.X[q]; v1 = P.V[q];
        }
        if (u0) pair(x0, v0);
        if (u1) pair(x1, v1);
      }
    } else {
      for (int k = 0; k < nmax; ++k) {
        int e = lr.get(k);
        if (k >= cnt) continue;
        int q = e & kSlotMask;
        pair(P.X[q], P.V[q]);
      }
    }
    if (active) {
      if (C1) {
        if (s.c1_be && s.c1_divu) {
          double B[9];
          load_b(P.BD, P.total_slots, p, B);
          b_renormalise(B, g1);
          b_renormalise(B, g2);
          b_renormalise(B, g3);
        }
        dden = dden - (g1[0] + g2[1] + g3[2]);
      } else if (DIM == 3) {
        dden = dden - (a1 + a2 + a3);
      } else {
        dden = dden - (a1 + a3);
      }
      if (FUSED) {
        // Leapfrog_continuity.f90:54-68, EoS_barotropic_linear.f90:49-55
        double rho = rhoi + dyn->dt * dden;
        if (s.density_thresholds == 1) {
          if (rho < 0.9 * s.den0) rho = 0.9 * s.den0;
          if (rho > 1.1 * s.den0) rho = 1.1 * s.den0;
        }
        double pr = s.k_over_rho0 * (rho - s.den0) + s.p_ref;
        P.RP[p] = make_double2(rho, pr);
      } else {
        P.DDEN[p] = dden;
      }
    }
  }
}

// ==========================================================================
// FP32-compensated form.  Pair arithmetic in FP32 on the screening copies
// (FP64 cell origin + FP32 offset) with compensated (Kahan) per-particle
// sums; the pressure term uses the symmetric form that the two accumulators
// of inter_EqMoto.f90:195-221 add up to.  Boundary terms, the elastic
// reaction, time integration and the time step stay in FP64.
// ==========================================================================
struct Kahan {
  float s, c;
  __device__ __forceinline__ void zero() {
    s = 0.f;
    c = 0.f;
  }
  // built without contraction (--fmad=false), as compensation requires
  __device__ __forceinline__ void add(float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double val() const { return (double)s - (double)c; }
};

struct F32Const {
  float hinv, h2inv, eta, eta2, ke, kacl, amon, nu, nu4;
  __device__ __forceinline__ void load(const SimDev& s) {
    hinv = (float)(1.0 / s.h);
    h2inv = (float)(1.0 / s.squareh);
    eta = (float)s.eta;
    eta2 = (float)s.eta2;
    ke = (float)s.ke_coef;
    kacl = (float)s.kacl_coef;
    amon = (float)(s.alfa_mon * (s.celerita + s.celerita) * s.h);
    nu = (float)s.kin_visc;
    nu4 = (float)(4.0 * (s.kin_visc * s.kin_visc));
  }
};

// The PTX approximate reciprocal and reciprocal square root (one special
// function unit instruction each, relative error about 2^-23, subnormals
// flushed): the FP32c pair terms' divisions and square roots.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Distance of a list pair from its squared distance: rr is positive for any
// two particles of distinct positions; the floor keeps r finite (0) should
// two FP32 offsets coincide.
__device__ __forceinline__ float pair_distance(float rr) {
  const float rq = fmaxf(rr, 1.0e-30f);
  return rq * rsqrt_approx(rq);
}

// Beta-spline gradient factors of a list pair (CalcVarLength.f90:230-262):
// PK1 = g ke / (r + eta), PK2 = PK1 / (rr + eta2), PK3 = gw kacl / (r + eta).
// The two divisions share one reciprocal: 1/a = b/(ab), 1/b = a/(ab).  A
// list pair has r <= 2h in FP64; its FP32 q may round a hair past 2, where
// both polynomials vanish to within rounding, so no support test is needed.
__device__ __forceinline__ void kernel_values_f32(const F32Const& c, float rr, float& PK1, float& PK2, float& PK3) {
  const float r = pair_distance(rr);
  const float q = r * c.hinv;
  const float q2 = rr * c.h2inv;
  const float a = r + c.eta, bq = rr + c.eta2;
  const float inv = rcp_approx(a * bq);
  const float denom = bq * inv;
  const float g = (q < 1.0f) ? fmaf(1.5f, q2, -2.0f * q) : fmaf(-0.5f, q2, fmaf(2.0f, q, -2.0f));
  const float gw = fmaf(12.0f, q, fmaf(-3.0f, q2, -12.0f));
  PK1 = g * c.ke * denom;
  PK2 = PK1 * (a * inv);
  PK3 = gw * c.kacl * denom;
}

// PK1 alone (the continuity pass).
__device__ __forceinline__ float kernel_pk1_f32(const F32Const& c, float rr) {
  const float r = pair_distance(rr);
  const float q = r * c.hinv;
  const float q2 = rr * c.h2inv;
  const float g = (q < 1.0f) ? fmaf(1.5f, q2, -2.0f * q) : fmaf(-0.5f, q2, fmaf(2.0f, q, -2.0f));
  return g * c.ke * rcp_approx(r + c.eta);
}

// Cell-origin offset of the neighbour column (run) a list entry names.  A
// lane's entries are stored run by run, so the offsets are formed again only
// when the run changes: (ci - ir) dcd = (1 - rx) dcd for the run's x column
// rx = r % 3 (r in 2D) and likewise in y.
template <int DIM>
struct RunCursor {
  int r = -1;
  float Dx = 0.f, Dy = 0.f;
  __device__ __forceinline__ void update(const SimDev& s, int run) {
    if (run == r) return;
    r = run;
    const int rx = (DIM == 3) ? run % 3 : run;
    Dx = (float)(1 - rx) * s.dcdf[0];
    Dy = (DIM == 3) ? (float)(1 - run / 3) * s.dcdf[1] : 0.f;
  }
};

// FP32 separation x_i - x_j of list entry e with neighbour record xj: the
// cell-origin difference (run offsets in x and y, (k_i - k_j) dcd in z, all
// exact small multiples) plus the offsets' difference.
template <int DIM>
__device__ __forceinline__ void separation_f32(const SimDev& s, RunCursor<DIM>& rc, int e, const float4& xj,
                                               const float4& xfi, float ckf, float dz, float& d0, float& d1,
                                               float& d2) {
  rc.update(s, (int)((unsigned)e >> kSlotBits));
  d0 = rc.Dx + (xfi.x - xj.x);
  d1 = (DIM == 3) ? rc.Dy + (xfi.y - xj.y) : 0.f;
  d2 = (ckf - xj.w) * dz + (xfi.z - xj.z);
}

// The closing of an FP32c momentum pass for particle p, from its nine pair
// sums ms and its FP64 wall terms (zero without close faces): the laminar
// flag (inter_EqMoto.f90:269-283), gravity, the elastic reaction, and in
// the fused step the leapfrog update and the particle's CFL time.  One
// function for both places a particle is closed (the finishing launch, and
// the pair launch itself for particles without close faces), so the two
// give the same bits.
template <int DIM, bool FUSED>
__device__ __forceinline__ void momentum_f32_close(const SimDev& s, const DevBatch& b, SimDyn* dyn, int p,
                                                   const double* ms, double* tpres, const double* tdiss,
                                                   const double* tvisc, const double* vi, double rhoi, double pi,
                                                   int nb, int bstart, double& dtc) {
  const Particles& P = b.P;
  const double GI = (double)9.80665f;   // Static_allocation_module.f90:72, a default-REAL literal
  const double* geff = dyn->geff;
  double rs0 = ms[6], rs1 = ms[7], rs2 = ms[8];
  tpres[0] = tpres[0] + ms[0];
  tpres[1] = tpres[1] + ms[1];
  tpres[2] = tpres[2] + ms[2];
  int lam_new = 0;
  if (s.kin_visc > 0.0) {
    double absv_pres = sqrt(tpres[0] * tpres[0] + tpres[1] * tpres[1] + tpres[2] * tpres[2]) + GI;
    double absv_morris = sqrt(rs0 * rs0 + rs1 * rs1 + rs2 * rs2);
    double weight = 0.0;
    if (absv_pres != 0.0) weight = absv_morris / absv_pres * 100.0;
    lam_new = (weight > 5.0 || absv_pres == 0.0) ? 1 : 0;
  }
  double acc[3];
  acc[0] = tpres[0] + (tdiss[0] + ms[3]) + (tvisc[0] + rs0) + geff[0];
  acc[1] = tpres[1] + (tdiss[1] + ms[4]) + (tvisc[1] + rs1) + geff[1];
  acc[2] = tpres[2] + (tdiss[2] + ms[5]) + (tvisc[2] + rs2) + geff[2];
  const double4 xi = P.X[p];
  if (nb > 0) {
    double R[3];
    const double xa[3] = {xi.x, xi.y, xi.z};
    elastic_reaction<DIM>(s, b, nb, bstart, xa, vi, R);
    for (int d = 0; d < 3; ++d) acc[d] = acc[d] + R[d];
  }
  if (FUSED) {
    double dtvel = dyn->dtvel, dt = dyn->dt;
    double vn[3];
    for (int d = 0; d < 3; ++d) vn[d] = vi[d] + dtvel * acc[d];
    P.X2[p] = make_double4(xi.x + dt * vn[0], xi.y + dt * vn[1], xi.z + dt * vn[2], xi.w);
    P.V2[p] = make_double4(vn[0], vn[1], vn[2], rhoi);
    if (P.VF2) P.VF2[p] = make_float4((float)vn[0], (float)vn[1], (float)vn[2], 0.f);
    P.P2[p] = pi;
    P.I2[p] = P.I[p];
    P.L2[p] = (uint8_t)lam_new;
    double U = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    // with velocity smoothing the CFL minimum is taken on the smoothed
    // velocities (k_velocity_smoothing_apply), which also moves X2
    if (!(s.teta_v > 1.0e-9)) dtc = s.cfl * 2.0 * s.h / (s.celerita + U);
  } else {
    P.ACC[p] = make_double4(acc[0], acc[1], acc[2], 0.0);
    P.L[p] = (uint8_t)lam_new;
  }
}

// Momentum, FP32c form, in two launches.  k_momentum_f32 holds only what
// the pair loop needs -- the particle's FP32 values, the compensated sums,
// the list chunk being read and the next one -- so that it runs at 3 blocks
// of 256 per SM without spilling (gathers are latency-bound: occupancy pays
// more than loading the next pair's records ahead), and writes the nine
// compensated sums of each particle to MSUM.
// k_momentum_f32_finish adds the FP64 wall terms (an independent sum), the
// laminar flag, gravity and the elastic reaction and, in the fused step,
// the leapfrog update and the CFL minimum.
// C1 (C1_BE): the pressure-gradient accumulator of inter_EqMoto.f90:195-204,
// -m_j (p_j - p_i) / (rho_i rho_j) PK3 r, is summed apart as well (the
// pressure difference formed in FP64), so the finishing launch can
// renormalise it with B_ren_gradp (inter_EqMoto.f90:255-260) and keep the
// ALE1 accumulator, the symmetric sum less it, as it is.
// BATCH: the twelve neighbour records of a list chunk are all requested
// before the first pair's arithmetic, four pairs' loads in flight per lane
// instead of one, at 2 blocks of 256 per SM (the registers they need); the
// autotuner chooses it or the lean loop (3 blocks per SM) on the live
// state.  Both sum the same terms in the same order: identical results.
// fused (the whole step, not C1): a particle without close faces has no
// FP64 wall terms, so this launch closes it at once (momentum_f32_close,
// the finishing launch's own code) instead of passing its nine sums on.
// PAIRED (with BATCH, not C1): two list entries' terms on Blackwell's paired
// FP32 instructions (pair2), the same bits as two calls of `pair`.
template <int DIM, bool C1 = false, bool BATCH = false, bool PAIRED = false>
__global__ void __launch_bounds__(kBlock, (C1 || BATCH) ? 2 : 3) k_momentum_f32(DevBatch b, int fused) {
  static_assert(!PAIRED || (BATCH && !C1), "the paired loop is a batched, non-C1 shape");
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    F32Const fc;
    fc.load(s);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen;
    int cnt = 0;
    float4 xfi = make_float4(0.f, 0.f, 0.f, 0.f);
    float vix = 0.f, viy = 0.f, viz = 0.f, rhof = 1.f, Pi = 0.f;
    double piD = 0.0;
    if (active) {
      double4 v4 = P.V[p];
      double2 rp = P.RP[p];
      xfi = P.XF[p];
      vix = (float)v4.x;
      viy = (float)v4.y;
      viz = (float)v4.z;
      rhof = (float)rp.x;
      Pi = (float)(rp.y / (rp.x * rp.x));
      piD = rp.y;
      cnt = b.ncount[p];
    }
    const float ckf = xfi.w, dz = s.dcdf[2];
    RunCursor<DIM> rc;
    const bool morris = s.kin_visc > 1.0e-12;
    // compensated sums of 4-entry partial sums (one list chunk each)
    Kahan tp0, tp1, tp2, td0, td1, td2, tv0, tv1, tv2;
    tp0.zero(); tp1.zero(); tp2.zero(); td0.zero(); td1.zero(); td2.zero(); tv0.zero(); tv1.zero(); tv2.zero();
    float cp0 = 0.f, cp1 = 0.f, cp2 = 0.f, cd0 = 0.f, cd1 = 0.f, cd2 = 0.f, cv0 = 0.f, cv1 = 0.f, cv2 = 0.f;
    Kahan tg0, tg1, tg2;
    tg0.zero(); tg1.zero(); tg2.zero();
    float cg0 = 0.f, cg1 = 0.f, cg2 = 0.f;
    // one list chunk (4 entries) per iteration: entries, compensation and
    // the next chunk's load handled once per chunk
    const int nch = (cnt + 3) >> 2;
    const int nchmax = __reduce_max_sync(0xffffffffu, (unsigned)nch);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nchmax * 4);
    const int4* lbase = reinterpret_cast<const int4*>(b.nlist) + list_base4(p, b.list_cap4);
    int4 nxt = nch > 0 ? __ldg(lbase) : make_int4(0, 0, 0, 0);
    // a neighbour's record is 40 B: XF (offset, cell k), VF (velocity,
    // m/rho) and RM (rho, p/rho^2); its mass is rho (m/rho)
    auto pair = [&](int e, const float4& xj, const float4& vj, const float2& rmj) {
      const int q = e & kSlotMask;
      float d0, d1, d2;
      separation_f32<DIM>(s, rc, e, xj, xfi, ckf, dz, d0, d1, d2);
      float rr = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      float PK1, PK2, PK3;
      kernel_values_f32(fc, rr, PK1, PK2, PK3);
      const float rhoj = rmj.x;
      const float mj = rhoj * vj.w;
      // pressure (both accumulators of inter_EqMoto together)
      float pf = -(mj * (Pi + rmj.y) * PK3);
      cp0 = fmaf(pf, d0, cp0);
      if (DIM == 3) cp1 = fmaf(pf, d1, cp1);
      cp2 = fmaf(pf, d2, cp2);
      if (C1) {
        const float dpf = (float)(__ldg(reinterpret_cast<const double*>(P.RP + q) + 1) - piD);
        const float gf = -(mj * dpf * rcp_approx(rhof * rhoj) * PK3);
        cg0 = fmaf(gf, d0, cg0);
        if (DIM == 3) cg1 = fmaf(gf, d1, cg1);
        cg2 = fmaf(gf, d2, cg2);
      }
      float dv0 = vj.x - vix, dv1 = vj.y - viy, dv2 = vj.z - viz;
      // viscomon amon / rsum and viscomorris nu4 / (nu rsum + 1e-3) from one
      // reciprocal of their denominators' product
      const float rsum = rhof + rhoj;
      const float bm = fmaf(fc.nu, rsum, 1.0e-3f);
      const float iv = rcp_approx(rsum * bm);
      float vr = -fmaf(dv2, d2, fmaf(dv1, d1, dv0 * d0));
      float df = mj * (fc.amon * (bm * iv)) * vr * PK2;
      cd0 = fmaf(df, d0, cd0);
      if (DIM == 3) cd1 = fmaf(df, d1, cd1);
      cd2 = fmaf(df, d2, cd2);
      if (morris) {
        float vf = -((mj * fc.nu4) * (rsum * iv) * PK2 * rr);
        cv0 = fmaf(vf, dv0, cv0);
        if (DIM == 3) cv1 = fmaf(vf, dv1, cv1);
        cv2 = fmaf(vf, dv2, cv2);
      }
    };
    // `pair` for entries ea, eb on paired instructions: every half rounds as
    // the scalar instruction does (x - y as fma(y, -1, x), one rounding
    // either way; products and sums in the scalar code's association, no
    // contraction), the special-function values, the cubic spline's branch
    // and the accumulations stay scalar, ea's accumulated before eb's.
    auto pair2 = [&](int ea, int eb, const float4& xa, const float4& va, const float2& ra, const float4& xb,
                     const float4& vb, const float2& rb) {
      const float2 m1 = make_float2(-1.f, -1.f);
      rc.update(s, (int)((unsigned)ea >> kSlotBits));
      const float dxa = rc.Dx, dya = rc.Dy;
      rc.update(s, (int)((unsigned)eb >> kSlotBits));
      const float2 Dx = make_float2(dxa, rc.Dx), Dy = make_float2(dya, rc.Dy);
      const float2 d0 = __fadd2_rn(Dx, __ffma2_rn(make_float2(xa.x, xb.x), m1, make_float2(xfi.x, xfi.x)));
      const float2 d1 = (DIM == 3) ? __fadd2_rn(Dy, __ffma2_rn(make_float2(xa.y, xb.y), m1, make_float2(xfi.y, xfi.y)))
                                   : make_float2(0.f, 0.f);
      const float2 dk = __ffma2_rn(make_float2(xa.w, xb.w), m1, make_float2(ckf, ckf));
      const float2 d2 = __fadd2_rn(__fmul2_rn(dk, make_float2(dz, dz)),
                                   __ffma2_rn(make_float2(xa.z, xb.z), m1, make_float2(xfi.z, xfi.z)));
      const float2 rr = __ffma2_rn(d2, d2, __ffma2_rn(d1, d1, __fmul2_rn(d0, d0)));
      // kernel_values_f32
      const float2 rq = make_float2(fmaxf(rr.x, 1.0e-30f), fmaxf(rr.y, 1.0e-30f));
      const float2 r = __fmul2_rn(rq, make_float2(rsqrt_approx(rq.x), rsqrt_approx(rq.y)));
      const float2 q = __fmul2_rn(r, make_float2(fc.hinv, fc.hinv));
      const float2 q2 = __fmul2_rn(rr, make_float2(fc.h2inv, fc.h2inv));
      const float2 a = __fadd2_rn(r, make_float2(fc.eta, fc.eta));
      const float2 bq = __fadd2_rn(rr, make_float2(fc.eta2, fc.eta2));
      const float2 ab = __fmul2_rn(a, bq);
      const float2 inv = make_float2(rcp_approx(ab.x), rcp_approx(ab.y));
      const float2 denom = __fmul2_rn(bq, inv);
      const float2 glo = __ffma2_rn(make_float2(1.5f, 1.5f), q2, __fmul2_rn(make_float2(-2.0f, -2.0f), q));
      const float2 ghi = __ffma2_rn(make_float2(-0.5f, -0.5f), q2,
                                    __ffma2_rn(make_float2(2.0f, 2.0f), q, make_float2(-2.0f, -2.0f)));
      const float2 g = make_float2(q.x < 1.0f ? glo.x : ghi.x, q.y < 1.0f ? glo.y : ghi.y);
      const float2 gw = __ffma2_rn(make_float2(12.0f, 12.0f), q,
                                   __ffma2_rn(make_float2(-3.0f, -3.0f), q2, make_float2(-12.0f, -12.0f)));
      const float2 PK1 = __fmul2_rn(__fmul2_rn(g, make_float2(fc.ke, fc.ke)), denom);
      const float2 PK2 = __fmul2_rn(PK1, __fmul2_rn(a, inv));
      const float2 PK3 = __fmul2_rn(__fmul2_rn(gw, make_float2(fc.kacl, fc.kacl)), denom);
      const float2 mj = __fmul2_rn(make_float2(ra.x, rb.x), make_float2(va.w, vb.w));
      // pressure: pf = -t
      const float2 t = __fmul2_rn(__fmul2_rn(mj, __fadd2_rn(make_float2(Pi, Pi), make_float2(ra.y, rb.y))), PK3);
      // viscosity
      const float2 dv0 = __ffma2_rn(make_float2(vix, vix), m1, make_float2(va.x, vb.x));
      const float2 dv1 = __ffma2_rn(make_float2(viy, viy), m1, make_float2(va.y, vb.y));
      const float2 dv2 = __ffma2_rn(make_float2(viz, viz), m1, make_float2(va.z, vb.z));
      const float2 rsum = __fadd2_rn(make_float2(rhof, rhof), make_float2(ra.x, rb.x));
      const float2 bm = __ffma2_rn(make_float2(fc.nu, fc.nu), rsum, make_float2(1.0e-3f, 1.0e-3f));
      const float2 rb2 = __fmul2_rn(rsum, bm);
      const float2 iv = make_float2(rcp_approx(rb2.x), rcp_approx(rb2.y));
      // vr = -u; df = -w
      const float2 u = __ffma2_rn(dv2, d2, __ffma2_rn(dv1, d1, __fmul2_rn(dv0, d0)));
      const float2 w = __fmul2_rn(
          __fmul2_rn(__fmul2_rn(mj, __fmul2_rn(make_float2(fc.amon, fc.amon), __fmul2_rn(bm, iv))), u), PK2);
      cp0 = fmaf(-t.x, d0.x, cp0);
      if (DIM == 3) cp1 = fmaf(-t.x, d1.x, cp1);
      cp2 = fmaf(-t.x, d2.x, cp2);
      cd0 = fmaf(-w.x, d0.x, cd0);
      if (DIM == 3) cd1 = fmaf(-w.x, d1.x, cd1);
      cd2 = fmaf(-w.x, d2.x, cd2);
      cp0 = fmaf(-t.y, d0.y, cp0);
      if (DIM == 3) cp1 = fmaf(-t.y, d1.y, cp1);
      cp2 = fmaf(-t.y, d2.y, cp2);
      cd0 = fmaf(-w.y, d0.y, cd0);
      if (DIM == 3) cd1 = fmaf(-w.y, d1.y, cd1);
      cd2 = fmaf(-w.y, d2.y, cd2);
      if (morris) {
        // vf = -z
        const float2 z = __fmul2_rn(
            __fmul2_rn(__fmul2_rn(__fmul2_rn(mj, make_float2(fc.nu4, fc.nu4)), __fmul2_rn(rsum, iv)), PK2), rr);
        cv0 = fmaf(-z.x, dv0.x, cv0);
        if (DIM == 3) cv1 = fmaf(-z.x, dv1.x, cv1);
        cv2 = fmaf(-z.x, dv2.x, cv2);
        cv0 = fmaf(-z.y, dv0.y, cv0);
        if (DIM == 3) cv1 = fmaf(-z.y, dv1.y, cv1);
        cv2 = fmaf(-z.y, dv2.y, cv2);
      }
    };
    for (int c = 0; c < nchmax; ++c) {
      const int4 ch = nxt;
      if (c + 1 < nch) nxt = __ldg(lbase + (size_t)(c + 1) * 32);
      if (c >= nch) continue;
      const int rem = cnt - 4 * c;   // >= 1
      if (BATCH) {
        float4 x0, v0, x1, v1, x2, v2, x3, v3;
        float2 r0, r1, r2, r3;
        const int q0 = ch.x & kSlotMask, q1 = ch.y & kSlotMask, q2 = ch.z & kSlotMask, q3 = ch.w & kSlotMask;
        x0 = __ldg(P.XF + q0); v0 = __ldg(P.VF + q0); r0 = __ldg(P.RM + q0);
        if (rem > 1) { x1 = __ldg(P.XF + q1); v1 = __ldg(P.VF + q1); r1 = __ldg(P.RM + q1); }
        if (rem > 2) { x2 = __ldg(P.XF + q2); v2 = __ldg(P.VF + q2); r2 = __ldg(P.RM + q2); }
        if (rem > 3) { x3 = __ldg(P.XF + q3); v3 = __ldg(P.VF + q3); r3 = __ldg(P.RM + q3); }
        if (PAIRED) {
          if (rem > 1) pair2(ch.x, ch.y, x0, v0, r0, x1, v1, r1);
          else pair(ch.x, x0, v0, r0);
          if (rem > 3) pair2(ch.z, ch.w, x2, v2, r2, x3, v3, r3);
          else if (rem > 2) pair(ch.z, x2, v2, r2);
        } else {
          pair(ch.x, x0, v0, r0);
          if (rem > 1) pair(ch.y, x1, v1, r1);
          if (rem > 2) pair(ch.z, x2, v2, r2);
          if (rem > 3) pair(ch.w, x3, v3, r3);
        }
      } else {
        auto one = [&](int e) {
          const int q = e & kSlotMask;
          pair(e, __ldg(P.XF + q), __ldg(P.VF + q), __ldg(P.RM + q));
        };
        one(ch.x);
        if (rem > 1) one(ch.y);
        if (rem > 2) one(ch.z);
        if (rem > 3) one(ch.w);
      }
      tp0.add(cp0); tp1.add(cp1); tp2.add(cp2);
      td0.add(cd0); td1.add(cd1); td2.add(cd2);
      tv0.add(cv0); tv1.add(cv1); tv2.add(cv2);
      cp0 = cp1 = cp2 = cd0 = cd1 = cd2 = cv0 = cv1 = cv2 = 0.f;
      if (C1) {
        tg0.add(cg0); tg1.add(cg1); tg2.add(cg2);
        cg0 = cg1 = cg2 = 0.f;
      }
    }
    bool close_here = false;
    if (!C1 && fused && active) close_here = P.bdt_count[p] == 0;
    double dtc = 1.0e300;
    if (close_here) {
      const double ms[9] = {tp0.val(), tp1.val(), tp2.val(), td0.val(), td1.val(), td2.val(),
                            tv0.val(), tv1.val(), tv2.val()};
      double tpres[3] = {0, 0, 0};
      const double tdiss[3] = {0, 0, 0}, tvisc[3] = {0, 0, 0};
      const double4 v4 = P.V[p];
      const double2 rp = P.RP[p];
      const double vi[3] = {v4.x, v4.y, v4.z};
      momentum_f32_close<DIM, true>(s, b, dyn, p, ms, tpres, tdiss, tvisc, vi, rp.x, rp.y, 0, 0, dtc);
    }
    if (!C1 && fused) {
      const double m = warp_min(dtc);
      if ((threadIdx.x & 31) == 0 && m < 1.0e300)
        atomicMin(&dyn->dtmin_bits, (unsigned long long)__double_as_longlong(m));
    }
    if (active && !close_here) {
      double* o = P.MSUM + p;
      const size_t st = (size_t)P.total_slots;   // component-major: coalesced
      o[0] = tp0.val();
      o[st] = tp1.val();
      o[2 * st] = tp2.val();
      o[3 * st] = td0.val();
      o[4 * st] = td1.val();
      o[5 * st] = td2.val();
      o[6 * st] = tv0.val();
      o[7 * st] = tv1.val();
      o[8 * st] = tv2.val();
      if (C1) {
        o[9 * st] = tg0.val();
        o[10 * st] = tg1.val();
        o[11 * st] = tg2.val();
      }
    }
  }
}

// C1: as the FP64 form (k_momentum<3, F, true>): the first step completes
// and inverts B_ren_gradp in the wall pass; the renormalised pressure-
// gradient accumulator joins the ALE1 accumulator and the wall terms.
template <int DIM, bool FUSED, bool C1 = false>
__global__ void __launch_bounds__(kBlock) k_momentum_f32_finish(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag;
    if (FUSED && active && dyn->frozen) {
      // a finished simulation of a batch: carry the record through the sort
      double4 v4 = P.V[p];
      double2 rp = P.RP[p];
      P.X2[p] = P.X[p];
      P.V2[p] = make_double4(v4.x, v4.y, v4.z, rp.x);
      P.P2[p] = rp.y;
      P.I2[p] = P.I[p];
      P.L2[p] = P.L[p];
      active = false;
    }
    double dtc = 1.0e300;
    // in the fused step the pair launch has closed the particles without
    // close faces already (k_momentum_f32)
    if (FUSED && !C1 && active && P.bdt_count[p] == 0) active = false;
    if (active) {
      double ms[9];
      for (int c = 0; c < 9; ++c) ms[c] = P.MSUM[(size_t)c * P.total_slots + p];
      double4 v4 = P.V[p];
      double2 rp = P.RP[p];
      const double vi[3] = {v4.x, v4.y, v4.z};
      const double rhoi = rp.x, pi = rp.y;
      const int nb = P.bdt_count[p];
      const int bstart = nb > 0 ? P.bdt_start[p] : 0;
      double tpres[3] = {0, 0, 0}, tdiss[3] = {0, 0, 0}, tvisc[3] = {0, 0, 0};
      const double* geff = dyn->geff;
      const bool c1 = C1 && DIM == 3 && s.c1_be;
      if (c1) {
        double B[9];
        const bool first = dyn->step == 0;
        load_b(P.BG, P.total_slots, p, B);
        if (nb > 0)
          me_boundary3d<true>(s, b, nb, bstart, vi, rhoi, pi, P.L[p], geff, tpres, tdiss, tvisc, B, first);
        else if (first)
          b_inversion(B, s.invb_det_thresh);
        if (first) store_b(P.BG, P.total_slots, p, B);
        // inter_EqMoto.f90:255-260: the pressure-gradient sum renormalised,
        // the ALE1 sum (the symmetric sum less it) as it is
        double g[3];
        for (int d = 0; d < 3; ++d) g[d] = P.MSUM[(size_t)(9 + d) * P.total_slots + p];
        const double al[3] = {ms[0] - g[0], ms[1] - g[1], ms[2] - g[2]};
        b_renormalise(B, g);
        for (int d = 0; d < 3; ++d) ms[d] = g[d] + al[d];
      } else if (nb > 0) {
        const int lam = P.L[p];
        if (DIM == 3) me_boundary3d(s, b, nb, bstart, vi, rhoi, pi, lam, geff, tpres, tdiss, tvisc);
        else me_boundary2d(s, b, nb, bstart, vi, rhoi, pi, lam, geff, tpres, tdiss, tvisc);
      }
      momentum_f32_close<DIM, FUSED>(s, b, dyn, p, ms, tpres, tdiss, tvisc, vi, rhoi, pi, nb, bstart, dtc);
    }
    if (FUSED) {
      double m = warp_min(dtc);
      if ((threadIdx.x & 31) == 0 && m < 1.0e300)
        atomicMin(&dyn->dtmin_bits, (unsigned long long)__double_as_longlong(m));
    }
  }
}

// Continuity, FP32c form, in two launches so that the pair sum need not
// wait for the boundary data: k_continuity_f32 writes the compensated pair
// sum of each particle to DDEN, and k_continuity_f32_finish, once the
// boundary data exist, forms dden = (SA-SPH wall term) - (pair sum) and, in
// the fused step, Leapfrog_continuity and the EoS.
// DIVU (C1_BE and C1_divu, 3D): a simulation that renormalises sums the
// whole velocity-gradient tensor, G(a, k) = sum rho_i (m_j / rho_j) PK1
// (v_j - v_i)_a r_k, nine compensated sums written to MSUM, which the
// finishing launch renormalises with B_ren_divu (Continuity_Equation.f90:
// 119-126,201-217); the others of the batch sum as without it.
// BATCH (not with DIVU): a list chunk's eight neighbour records requested
// before the chunk's arithmetic, at 3 blocks per SM; the same sums.
// PAIRED (with BATCH): two entries' terms on paired FP32 instructions
// (contrib2), the same bits as two calls of `contrib`.
template <int DIM, bool DIVU = false, bool BATCH = false, bool PAIRED = false>
__global__ void __launch_bounds__(kBlock, DIVU ? 2 : (BATCH ? 3 : 5)) k_continuity_f32(DevBatch b) {
  static_assert(!PAIRED || (BATCH && !DIVU), "the paired loop is a batched, non-C1 shape");
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    F32Const fc;
    fc.load(s);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen;
    int cnt = 0;
    float4 xfi = make_float4(0.f, 0.f, 0.f, 0.f);
    float vix = 0.f, viy = 0.f, viz = 0.f, rhof = 1.f;
    if (active) {
      double4 vi = P.V[p];
      xfi = P.XF[p];
      vix = (float)vi.x;
      viy = (float)vi.y;
      viz = (float)vi.z;
      rhof = (float)P.RP[p].x;
      cnt = b.ncount[p];
    }
    const float ckf = xfi.w, dz = s.dcdf[2];
    RunCursor<DIM> rc;
    const bool tensor = DIVU && DIM == 3 && s.c1_be && s.c1_divu;
    Kahan sum;
    sum.zero();
    float part = 0.f;   // 4-entry partial sum, compensated into sum per chunk
    Kahan gs[9];
    float gp[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      gs[a].zero();
      gp[a] = 0.f;
    }
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    if (BATCH && !DIVU) {
      auto contrib = [&](int e, const float4& xj, const float4& vj) {
        float d0, d1, d2;
        separation_f32<DIM>(s, rc, e, xj, xfi, ckf, dz, d0, d1, d2);
        float rr = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
        const float PK1 = kernel_pk1_f32(fc, rr);
        float c = rhof * vj.w * PK1;
        part = fmaf(c, fmaf(vj.z - viz, d2, fmaf(vj.y - viy, d1, (vj.x - vix) * d0)), part);
      };
      // contrib for entries ea, eb on paired instructions (each half rounds
      // as the scalar instruction; x - y as fma(y, -1, x)), ea's term
      // accumulated before eb's
      auto contrib2 = [&](int ea, int eb, const float4& xa, const float4& va, const float4& xb, const float4& vb) {
        const float2 m1 = make_float2(-1.f, -1.f);
        rc.update(s, (int)((unsigned)ea >> kSlotBits));
        const float dxa = rc.Dx, dya = rc.Dy;
        rc.update(s, (int)((unsigned)eb >> kSlotBits));
        const float2 Dx = make_float2(dxa, rc.Dx), Dy = make_float2(dya, rc.Dy);
        const float2 d0 = __fadd2_rn(Dx, __ffma2_rn(make_float2(xa.x, xb.x), m1, make_float2(xfi.x, xfi.x)));
        const float2 d1 = (DIM == 3)
                              ? __fadd2_rn(Dy, __ffma2_rn(make_float2(xa.y, xb.y), m1, make_float2(xfi.y, xfi.y)))
                              : make_float2(0.f, 0.f);
        const float2 dk = __ffma2_rn(make_float2(xa.w, xb.w), m1, make_float2(ckf, ckf));
        const float2 d2 = __fadd2_rn(__fmul2_rn(dk, make_float2(dz, dz)),
                                     __ffma2_rn(make_float2(xa.z, xb.z), m1, make_float2(xfi.z, xfi.z)));
        const float2 rr = __ffma2_rn(d2, d2, __ffma2_rn(d1, d1, __fmul2_rn(d0, d0)));
        // kernel_pk1_f32
        const float2 rq = make_float2(fmaxf(rr.x, 1.0e-30f), fmaxf(rr.y, 1.0e-30f));
        const float2 r = __fmul2_rn(rq, make_float2(rsqrt_approx(rq.x), rsqrt_approx(rq.y)));
        const float2 q = __fmul2_rn(r, make_float2(fc.hinv, fc.hinv));
        const float2 q2 = __fmul2_rn(rr, make_float2(fc.h2inv, fc.h2inv));
        const float2 glo = __ffma2_rn(make_float2(1.5f, 1.5f), q2, __fmul2_rn(make_float2(-2.0f, -2.0f), q));
        const float2 ghi = __ffma2_rn(make_float2(-0.5f, -0.5f), q2,
                                      __ffma2_rn(make_float2(2.0f, 2.0f), q, make_float2(-2.0f, -2.0f)));
        const float2 g = make_float2(q.x < 1.0f ? glo.x : ghi.x, q.y < 1.0f ? glo.y : ghi.y);
        const float2 ra = __fadd2_rn(r, make_float2(fc.eta, fc.eta));
        const float2 PK1 = __fmul2_rn(__fmul2_rn(g, make_float2(fc.ke, fc.ke)),
                                      make_float2(rcp_approx(ra.x), rcp_approx(ra.y)));
        const float2 c = __fmul2_rn(__fmul2_rn(make_float2(rhof, rhof), make_float2(va.w, vb.w)), PK1);
        const float2 dv0 = __ffma2_rn(make_float2(vix, vix), m1, make_float2(va.x, vb.x));
        const float2 dv1 = __ffma2_rn(make_float2(viy, viy), m1, make_float2(va.y, vb.y));
        const float2 dv2 = __ffma2_rn(make_float2(viz, viz), m1, make_float2(va.z, vb.z));
        const float2 u = __ffma2_rn(dv2, d2, __ffma2_rn(dv1, d1, __fmul2_rn(dv0, d0)));
        part = fmaf(c.x, u.x, part);
        part = fmaf(c.y, u.y, part);
      };
      const int nch = (cnt + 3) >> 2, nchmax = (nmax + 3) >> 2;
      const int4* lbase = reinterpret_cast<const int4*>(b.nlist) + list_base4(p, b.list_cap4);
      int4 nxt = nch > 0 ? __ldg(lbase) : make_int4(0, 0, 0, 0);
      for (int c = 0; c < nchmax; ++c) {
        const int4 ch = nxt;
        if (c + 1 < nch) nxt = __ldg(lbase + (size_t)(c + 1) * 32);
        if (c >= nch) continue;
        const int rem = cnt - 4 * c;
        const int q0 = ch.x & kSlotMask, q1 = ch.y & kSlotMask, q2 = ch.z & kSlotMask, q3 = ch.w & kSlotMask;
        float4 x0, v0, x1, v1, x2, v2, x3, v3;
        x0 = __ldg(P.XF + q0); v0 = __ldg(P.VF + q0);
        if (rem > 1) { x1 = __ldg(P.XF + q1); v1 = __ldg(P.VF + q1); }
        if (rem > 2) { x2 = __ldg(P.XF + q2); v2 = __ldg(P.VF + q2); }
        if (rem > 3) { x3 = __ldg(P.XF + q3); v3 = __ldg(P.VF + q3); }
        if (PAIRED) {
          if (rem > 1) contrib2(ch.x, ch.y, x0, v0, x1, v1);
          else contrib(ch.x, x0, v0);
          if (rem > 3) contrib2(ch.z, ch.w, x2, v2, x3, v3);
          else if (rem > 2) contrib(ch.z, x2, v2);
        } else {
          contrib(ch.x, x0, v0);
          if (rem > 1) contrib(ch.y, x1, v1);
          if (rem > 2) contrib(ch.z, x2, v2);
          if (rem > 3) contrib(ch.w, x3, v3);
        }
        sum.add(part);
        part = 0.f;
      }
    }
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, (BATCH && !DIVU) ? 0 : cnt);
    for (int k = 0; k < ((BATCH && !DIVU) ? 0 : nmax); ++k) {
      const int e = lr.get(k);
      if (k >= cnt) continue;
      const float4 xj = __ldg(P.XF + (e & kSlotMask)), vj = __ldg(P.VF + (e & kSlotMask));
      float d0, d1, d2;
      separation_f32<DIM>(s, rc, e, xj, xfi, ckf, dz, d0, d1, d2);
      float rr = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      const float PK1 = kernel_pk1_f32(fc, rr);
      float c = rhof * vj.w * PK1;    // rho_i (m_j / rho_j) PK1
      const bool flush = (k & 3) == 3 || k == cnt - 1;
      if (DIVU && tensor) {
        const float cv[3] = {c * (vj.x - vix), c * (vj.y - viy), c * (vj.z - viz)};
        const float dd[3] = {d0, d1, d2};
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
          for (int q = 0; q < 3; ++q) gp[3 * a + q] = fmaf(cv[a], dd[q], gp[3 * a + q]);
        if (flush) {
#pragma unroll
          for (int a = 0; a < 9; ++a) {
            gs[a].add(gp[a]);
            gp[a] = 0.f;
          }
        }
      } else {
        part = fmaf(c, fmaf(vj.z - viz, d2, fmaf(vj.y - viy, d1, (vj.x - vix) * d0)), part);
        if (flush) {
          sum.add(part);
          part = 0.f;
        }
      }
    }
    if (active) {
      if (DIVU && tensor) {
#pragma unroll
        for (int a = 0; a < 9; ++a) P.MSUM[(size_t)a * P.total_slots + p] = gs[a].val();
      } else {
        P.DDEN[p] = sum.val();
      }
    }
  }
}

// C1 (3D): the frontiers complete both matrices, which are inverted for
// every particle (continuity_boundary_c1, FP64); with C1_divu the pair
// tensor is renormalised with B_ren_divu and its trace enters drho/dt.
template <int DIM, bool FUSED, bool C1 = false>
__global__ void __launch_bounds__(kBlock) k_continuity_f32_finish(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    if (!(threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen)) continue;
    const double4 vi = P.V[p];
    const double rhoi = P.RP[p].x;
    double dden = 0.0;
    const int nb = P.bdt_count[p];
    if (C1 && DIM == 3 && s.c1_be) {
      dden = continuity_boundary_c1(s, b, dyn, nb, nb > 0 ? P.bdt_start[p] : 0, vi, rhoi, p);
      if (s.c1_divu) {
        double B[9], g[3][3];
        load_b(P.BD, P.total_slots, p, B);
        for (int a = 0; a < 3; ++a) {
          for (int q = 0; q < 3; ++q) g[a][q] = P.MSUM[(size_t)(3 * a + q) * P.total_slots + p];
          b_renormalise(B, g[a]);
        }
        dden = dden - (g[0][0] + g[1][1] + g[2][2]);
      } else {
        dden = dden - P.DDEN[p];
      }
    } else {
      if (nb > 0) dden = continuity_boundary<DIM>(s, b, dyn, nb, P.bdt_start[p], vi, rhoi);
      dden = dden - P.DDEN[p];
    }
    if (FUSED) {
      double rho = rhoi + dyn->dt * dden;
      if (s.density_thresholds == 1) {
        if (rho < 0.9 * s.den0) rho = 0.9 * s.den0;
        if (rho > 1.1 * s.den0) rho = 1.1 * s.den0;
      }
      double pr = s.k_over_rho0 * (rho - s.den0) + s.p_ref;
      P.RP[p] = make_double2(rho, pr);
      const double m = P.X[p].w;
      P.RF[p] = make_float4((float)rho, (float)(pr / (rho * rho)), (float)m, 0.f);
      // the next momentum pass's records: the new density, and m/rho in
      // VF.w (the pair sums of this pass, which read the old one, are done)
      P.RM[p] = make_float2((float)rho, (float)(pr / (rho * rho)));
      P.VF[p].w = (float)(m / rho);
    } else {
      P.DDEN[p] = dden;
    }
  }
}

// FP32 copies of velocity, density and pressure after an in-place update
// of the FP64 state by the per-call ABI.
__global__ void k_refresh_f32(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    double4 x = b.P.X[p];
    double4 v = b.P.V[p];
    double2 rp = b.P.RP[p];
    // m/rho of the current density (after a pressure smoothing V.w still
    // holds the sort's; where they agree this is the same division)
    b.P.VF[p] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)(x.w / rp.x));
    b.P.RF[p] = make_float4((float)rp.x, (float)(rp.y / (rp.x * rp.x)), (float)x.w, 0.f);
    b.P.RM[p] = make_float2((float)rp.x, (float)(rp.y / (rp.x * rp.x)));
  }
}

// ==========================================================================
// Partial smoothing (input_any_t%TetaV, %TetaP > 0), FP64 in both forms.
// The reference's neighbour list includes the particle itself; the lists
// here leave it out, so its term is added where the reference's order puts
// it: before the first entry past (centre run, own slot).
// ==========================================================================

// PartKernel(4) of CalcVarLength.f90:241-268: the kernel value W = wu coefke.
__device__ __forceinline__ double kernel_w(const SimDev& s, double rr) {
  double r = sqrt(rr);
  double q = div_rn(r, s.h, s.rcp_h);
  double q2 = div_rn(rr, s.squareh, s.rcp_squareh);
  int idx = (int)q;
  if (idx >= 2) return 0.0;
  double wu = 0.666666667 + q2 * (q * 0.5 - 1.0);
  if (idx > 0) wu = (2.0 - q) * (2.0 - q) * (2.0 - q) * 0.166666666667;
  return wu * s.coefke;
}

// velocity_smoothing_SA_SPH_3D.f90:61-125 / _2D.f90:66-117 (fixe/tapi
// walls, slip mode 1): adds the wall terms of particle p to var.
template <int DIM>
__device__ __forceinline__ void smoothing_wall_velocity(const SimDev& s, const DevBatch& b, int p, const double4& vi,
                                                        double* var) {
  const Particles& P = b.P;
  const int nb = P.bdt_count[p];
  const int bstart = nb > 0 ? P.bdt_start[p] : 0;
  for (int u = 0; u < nb; ++u) {
    const BdtEntry& e = P.bdt[bstart + u];
    if (DIM == 3) {
      const FaceDev& f = b.faces[s.face_off + e.clobonum - 1];
      const double vv[3] = {vi.x, vi.y, vi.z};
      double DVGlo[3], DVLoc[3], BCLoc[3];
      for (int i = 0; i < 3; ++i) DVGlo[i] = 2.0 * (f.velocity[i] - vv[i]);
      for (int i = 0; i < 3; ++i) {
        double a = 0.0;
        for (int j = 0; j < 3; ++j) a = a + f.T[j][i] * DVGlo[j];
        DVLoc[i] = a;
      }
      double IntWdV = e.bi[1];
      BCLoc[0] = DVLoc[0] * IntWdV * f.slip;
      BCLoc[1] = DVLoc[1] * IntWdV * f.slip;
      BCLoc[2] = DVLoc[2] * IntWdV;
      for (int i = 0; i < 3; ++i) {
        double g = 0.0;
        for (int j = 0; j < 3; ++j) g = g + f.T[i][j] * BCLoc[j];
        var[i] = var[i] + g;
      }
    } else {
      const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
      double DVGlo0 = 2.0 * (S.velocity[0] - vi.x), DVGlo1 = 2.0 * (S.velocity[2] - vi.z);
      double DVLoc0 = S.sss[0] * DVGlo0 + S.sss[1] * DVGlo1;
      double DVLoc1 = S.nnn[0] * DVGlo0 + S.nnn[1] * DVGlo1;
      double IntWdV = e.bi[2];
      double BCLoc0 = DVLoc0 * IntWdV * S.slip;
      double BCLoc1 = DVLoc1 * IntWdV;
      var[0] = var[0] + (S.sss[0] * BCLoc0 + S.nnn[0] * BCLoc1);
      var[2] = var[2] + (S.sss[1] * BCLoc0 + S.nnn[1] * BCLoc1);
    }
  }
}

// The wall terms and the update of PressureSmoothing_3D.f90:111-134 /
// _2D.f90:140-212 for particle p with pair sums sompW and AppUnity: the
// smoothed pressure.
template <int DIM>
__device__ __forceinline__ double smoothing_pressure(const SimDev& s, const DevBatch& b, const SimDyn* dyn, int p,
                                                     double pi, double sompW, double AppUnity) {
  const Particles& P = b.P;
  const double TetaP1 = s.teta_p * s.celerita * dyn->dt / s.h;
  const double p0i = s.p_ref;
  const int nb = P.bdt_count[p];
  const int bstart = nb > 0 ? P.bdt_start[p] : 0;
  double vpres;
  if (DIM == 3) {
    for (int u = 0; u < nb; ++u) {
      const BdtEntry& e = P.bdt[bstart + u];
      if (e.loc[2] > 0.0) AppUnity = AppUnity + e.bi[1];
    }
    double DiffP = (AppUnity < 0.95) ? sompW + (p0i - pi) * (1.0 - AppUnity) : sompW / AppUnity;
    vpres = pi + TetaP1 * DiffP;
  } else {
    const double* g = dyn->geff;
    double VIntWdV_FT = 0.0;
    for (int u = 0; u < nb; ++u) {
      const BdtEntry& e = P.bdt[bstart + u];
      const SideDev& S = b.sides[s.side_off + e.clobonum - 1];
      double mf0 = S.sss[0] * g[0] + S.sss[1] * g[2];
      double mf1 = S.nnn[0] * g[0] + S.nnn[1] * g[2];
      VIntWdV_FT = VIntWdV_FT + e.bi[1];
      sompW = sompW + s.den0 * (mf0 * e.bi[3] + mf1 * e.bi[4]);
    }
    AppUnity = AppUnity + VIntWdV_FT + 0.0 + 0.0 + 0.0;
    vpres = pi + TetaP1 * (sompW + (pi - pi) * 0.0 + (pi - pi) * 0.0 + (p0i - pi) * (1.0 - AppUnity));
  }
  return vpres;
}

// velocity_smoothing.f90:85-132 with velocity_smoothing_SA_SPH_3D.f90:61-125
// / _2D.f90:66-117 (fixe/tapi walls, slip mode 1): ACC = var, the smoothing
// increment, from the velocities `vel` (the step's leapfrog velocities).
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_velocity_smoothing(DevBatch b, const double4* __restrict__ vel) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  constexpr int RC = (DIM == 3) ? 4 : 1;   // the particle's own column run
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_v > 1.0e-9;
    const int cnt = active ? b.ncount[p] : 0;
    double var[3] = {0.0, 0.0, 0.0};
    double4 xi = make_double4(0.0, 0.0, 0.0, 0.0), vi = xi;
    double self_w = 0.0;
    if (active) {
      xi = P.X[p];
      vi = vel[p];
      self_w = xi.w * kernel_w(s, 0.0) / P.RP[p].x;
    }
    bool self_done = !active;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    for (int k = 0; k < nmax; ++k) {
      int e = lr.get(k);
      if (k >= cnt) continue;
      int q = e & kSlotMask;
      int r = (int)((unsigned)e >> kSlotBits);
      if (!self_done && (r > RC || (r == RC && q > p))) {
        var[0] = var[0] + (vi.x - vi.x) * self_w;
        var[1] = var[1] + (vi.y - vi.y) * self_w;
        var[2] = var[2] + (vi.z - vi.z) * self_w;
        self_done = true;
      }
      double4 xj = P.X[q];
      double r0 = xi.x - xj.x, r1 = xi.y - xj.y, r2 = xi.z - xj.z;
      double rr = r0 * r0 + r1 * r1 + r2 * r2;
      double pesoj = xj.w * kernel_w(s, rr) / P.RP[q].x;
      double4 vj = vel[q];
      var[0] = var[0] + (vj.x - vi.x) * pesoj;
      var[1] = var[1] + (vj.y - vi.y) * pesoj;
      var[2] = var[2] + (vj.z - vi.z) * pesoj;
    }
    if (!active) continue;
    if (!self_done) {
      var[0] = var[0] + (vi.x - vi.x) * self_w;
      var[1] = var[1] + (vi.y - vi.y) * self_w;
      var[2] = var[2] + (vi.z - vi.z) * self_w;
    }
    smoothing_wall_velocity<DIM>(s, b, p, vi, var);
    P.ACC[p] = make_double4(var[0], var[1], var[2], 0.0);
  }
}

// The FP32c form's smoothing sums: the same terms in FP32 from the FP32
// records (XF, RF, and VF2, the leapfrog velocities the momentum pass
// writes in FP32) with compensated 4-entry chunk sums, the pressure
// differences formed in FP64 first; the particle's own term (zero for
// velocities) and the wall terms in FP64.
__device__ __forceinline__ float kernel_w_f32(float rr, float hinv, float coefke) {
  float r = rr * rsqrtf(rr);
  float q = r * hinv;
  if (!(q < 2.0f)) return 0.f;
  float wu = (q < 1.0f) ? fmaf(q * q, fmaf(q, 0.5f, -1.0f), 0.666666667f)
                        : (2.0f - q) * (2.0f - q) * (2.0f - q) * (1.0f / 6.0f);
  return wu * coefke;
}

template <int DIM>
__global__ void __launch_bounds__(kBlock, 4) k_velocity_smoothing_f32(DevBatch b, const double4* __restrict__ vel) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_v > 1.0e-9;
    const float hinv = (float)(1.0 / s.h), coefke = (float)s.coefke;
    int cnt = 0;
    float4 xfi = make_float4(0.f, 0.f, 0.f, 0.f);
    double4 vi = make_double4(0.0, 0.0, 0.0, 0.0);
    if (active) {
      xfi = P.XF[p];
      vi = vel[p];
      cnt = b.ncount[p];
    }
    const float ckf = xfi.w, dz = s.dcdf[2];
    RunCursor<DIM> rc;
    const float4 vif = make_float4((float)vi.x, (float)vi.y, (float)vi.z, 0.f);
    Kahan k0, k1, k2;
    k0.zero(); k1.zero(); k2.zero();
    float c0 = 0.f, c1 = 0.f, c2 = 0.f;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    for (int k = 0; k < nmax; ++k) {
      int e = lr.get(k);
      if (k >= cnt) continue;
      int q = e & kSlotMask;
      const float4 xj = P.XF[q], rfj = P.RF[q], vj = P.VF2[q];
      float d0, d1, d2;
      separation_f32<DIM>(s, rc, e, xj, xfi, ckf, dz, d0, d1, d2);
      float rr = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      float pes = __fdividef(rfj.z * kernel_w_f32(rr, hinv, coefke), rfj.x);
      c0 = fmaf(vj.x - vif.x, pes, c0);
      if (DIM == 3) c1 = fmaf(vj.y - vif.y, pes, c1);
      c2 = fmaf(vj.z - vif.z, pes, c2);
      if ((k & 3) == 3 || k == cnt - 1) {
        k0.add(c0); k1.add(c1); k2.add(c2);
        c0 = c1 = c2 = 0.f;
      }
    }
    if (!active) continue;
    double var[3] = {k0.val(), k1.val(), k2.val()};
    smoothing_wall_velocity<DIM>(s, b, p, vi, var);
    P.ACC[p] = make_double4(var[0], var[1], var[2], 0.0);
  }
}

template <int DIM>
__global__ void __launch_bounds__(kBlock, 4) k_pressure_smoothing_f32(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_p > 0.0;
    const float hinv = (float)(1.0 / s.h), coefke = (float)s.coefke;
    int cnt = 0;
    float4 xfi = make_float4(0.f, 0.f, 0.f, 0.f);
    double pi = 0.0;
    float self = 0.f;
    if (active) {
      xfi = P.XF[p];
      const float4 rfi = P.RF[p];
      pi = P.RP[p].y;
      self = __fdividef(rfi.z * (0.666666667f * coefke), rfi.x);
      cnt = b.ncount[p];
    }
    const float ckf = xfi.w, dz = s.dcdf[2];
    RunCursor<DIM> rc;
    Kahan ka, ks;
    ka.zero();
    ks.zero();
    float ca = self, cs = 0.f;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    for (int k = 0; k < nmax; ++k) {
      int e = lr.get(k);
      if (k >= cnt) continue;
      int q = e & kSlotMask;
      const float4 xj = P.XF[q], rfj = P.RF[q];
      const float dp = (float)(P.RP[q].y - pi);
      float d0, d1, d2;
      separation_f32<DIM>(s, rc, e, xj, xfi, ckf, dz, d0, d1, d2);
      float rr = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
      float pes = __fdividef(rfj.z * kernel_w_f32(rr, hinv, coefke), rfj.x);
      ca += pes;
      cs = fmaf(dp, pes, cs);
      if ((k & 3) == 3 || k == cnt - 1) {
        ka.add(ca);
        ks.add(cs);
        ca = cs = 0.f;
      }
    }
    if (!active) continue;
    if (cnt == 0) ka.add(ca);   // the particle's own term alone
    P.DDEN[p] = smoothing_pressure<DIM>(s, b, dyn, p, pi, ks.val(), ka.val());
  }
}

// velocity_smoothing_2.f90:87-101 with TetaV > 1e-9: vel = vel + TetaV1 var.
// FUSED (the step graph): on the momentum pass's record V2, then
// Leapfrog_trajectories into X2 and the CFL minimum of the smoothed
// velocities; otherwise in place on V (the per-call ABI).
template <bool FUSED>
__global__ void __launch_bounds__(kBlock) k_velocity_smoothing_apply(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_v > 1.0e-9;
    double dtc = 1.0e300;
    if (active) {
      const double TetaV1 = s.teta_v * s.celerita * dyn->dt / s.h;
      const double4 var = P.ACC[p];
      double4 v = FUSED ? P.V2[p] : P.V[p];
      v.x = v.x + TetaV1 * var.x;
      v.y = v.y + TetaV1 * var.y;
      v.z = v.z + TetaV1 * var.z;
      if (FUSED) {
        P.V2[p] = v;
        const double4 x = P.X[p];
        const double dt = dyn->dt;
        P.X2[p] = make_double4(x.x + dt * v.x, x.y + dt * v.y, x.z + dt * v.z, x.w);
        double U = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
        dtc = s.cfl * 2.0 * s.h / (s.celerita + U);
      } else {
        P.V[p] = v;
      }
    }
    if (FUSED) {
      double m = warp_min(dtc);
      if ((threadIdx.x & 31) == 0 && m < 1.0e300)
        atomicMin(&dyn->dtmin_bits, (unsigned long long)__double_as_longlong(m));
    }
  }
}

// PressureSmoothing_3D.f90:88-134 / PressureSmoothing_2D.f90:102-212
// (SmoothVersion "b", fixe/tapi walls): DDEN = the smoothed pressure, from
// the pressures and densities after the step's EoS.
template <int DIM>
__global__ void __launch_bounds__(kBlock) k_pressure_smoothing(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  constexpr int RC = (DIM == 3) ? 4 : 1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    const bool active = threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_p > 0.0;
    const int cnt = active ? b.ncount[p] : 0;
    double4 xi = make_double4(0.0, 0.0, 0.0, 0.0);
    double pi = 0.0, self_w = 0.0, sompW = 0.0, AppUnity = 0.0;
    if (active) {
      xi = P.X[p];
      double2 rp = P.RP[p];
      pi = rp.y;
      self_w = xi.w * kernel_w(s, 0.0) / rp.x;
    }
    bool self_done = !active;
    ListPrefetcher lr;
    lr.init(b.nlist, p, b.list_cap4, cnt);
    const int nmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    prefetch_list_l2(b.nlist, p, b.list_cap4, nmax);
    for (int k = 0; k < nmax; ++k) {
      int e = lr.get(k);
      if (k >= cnt) continue;
      int q = e & kSlotMask;
      int r = (int)((unsigned)e >> kSlotBits);
      if (!self_done && (r > RC || (r == RC && q > p))) {
        AppUnity = AppUnity + self_w;
        sompW = sompW + (pi - pi) * self_w;
        self_done = true;
      }
      double4 xj = P.X[q];
      double r0 = xi.x - xj.x, r1 = xi.y - xj.y, r2 = xi.z - xj.z;
      double rr = r0 * r0 + r1 * r1 + r2 * r2;
      double2 rpj = P.RP[q];
      double pesoj = xj.w * kernel_w(s, rr) / rpj.x;
      AppUnity = AppUnity + pesoj;
      sompW = sompW + (rpj.y - pi) * pesoj;
    }
    if (!active) continue;
    if (!self_done) {
      AppUnity = AppUnity + self_w;
      sompW = sompW + (pi - pi) * self_w;
    }
    P.DDEN[p] = smoothing_pressure<DIM>(s, b, dyn, p, pi, sompW, AppUnity);
  }
}

// PressureSmoothing_3D.f90:137-158 / _2D.f90:216-233: p = the smoothed
// pressure, density from the inverse EoS (EoS_barotropic_linear.f90:54),
// and the FP32 record of the FP32c form.
__global__ void __launch_bounds__(kBlock) k_pressure_smoothing_apply(DevBatch b, int refresh_f32) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    SimDyn* dyn = b.dyn + tl.sim;
    int p = tl.start + threadIdx.x;
    if (!(threadIdx.x < tl.count && p < s.p_off + dyn->nag && !dyn->frozen && s.teta_p > 0.0)) continue;
    double pr = P.DDEN[p];
    double rho = s.den0 * (1.0 + (pr - s.p_ref) / s.eps);
    P.RP[p] = make_double2(rho, pr);
    if (refresh_f32) {
      const double m = P.X[p].w;
      P.RF[p] = make_float4((float)rho, (float)(pr / (rho * rho)), (float)m, 0.f);
      P.RM[p] = make_float2((float)rho, (float)(pr / (rho * rho)));
      P.VF[p].w = (float)(m / rho);
    }
  }
}

// ==========================================================================
// Fine-grained integration kernels (used by the per-call C ABI)
// ==========================================================================
__global__ void k_leapfrog_momentum(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    double dtvel = b.dyn[tl.sim].dtvel;
    double4 v = b.P.V[p];
    double4 a = b.P.ACC[p];
    v.x = v.x + dtvel * a.x;
    v.y = v.y + dtvel * a.y;
    v.z = v.z + dtvel * a.z;
    b.P.V[p] = v;
    if (b.P.VF2) b.P.VF2[p] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
  }
}

__global__ void k_leapfrog_trajectories(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    double dt = b.dyn[tl.sim].dt;
    double4 x = b.P.X[p];
    double4 v = b.P.V[p];
    x.x = x.x + dt * v.x;
    x.y = x.y + dt * v.y;
    x.z = x.z + dt * v.z;
    b.P.X[p] = x;   // the screening copies are rebuilt by the next sph_ord_grid
  }
}

__global__ void k_leapfrog_continuity(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    double2 rp = b.P.RP[p];
    double rho = rp.x + b.dyn[tl.sim].dt * b.P.DDEN[p];
    if (s.density_thresholds == 1) {
      if (rho < 0.9 * s.den0) rho = 0.9 * s.den0;
      if (rho > 1.1 * s.den0) rho = 1.1 * s.den0;
    }
    b.P.RP[p] = make_double2(rho, rp.y);
    double4 v = b.P.V[p];
    v.w = b.P.X[p].w / rho;
    b.P.V[p] = v;
  }
}

__global__ void k_eos(DevBatch b) {
  __shared__ SimDev s;
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    if (b.dyn[tl.sim].step < 0) continue;   // EoS_fluid_loop.f90:61 (on_going_time_step > 0)
    double2 rp = b.P.RP[p];
    rp.y = s.k_over_rho0 * (rp.x - s.den0) + s.p_ref;
    b.P.RP[p] = rp;
  }
}

// CFL minimum of time_step_duration.f90:86-110 over the current velocities.
__global__ void k_dt_reduce(DevBatch b) {
  __shared__ SimDev s;
  __shared__ double red[kBlock / 32];
  int cur = -1;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    double dtc = 1.0e300;
    if (threadIdx.x < tl.count && p < s.p_off + b.dyn[tl.sim].nag) {
      double4 v = b.P.V[p];
      double U = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
      dtc = s.cfl * 2.0 * s.h / (s.celerita + U);
    }
    double m = warp_min(dtc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = red[0];
      for (int w = 1; w < kBlock / 32; ++w) mm = fmin(mm, red[w]);
      if (mm < 1.0e300) atomicMin(&b.dyn[tl.sim].dtmin_bits, (unsigned long long)__double_as_longlong(mm));
    }
    __syncthreads();
  }
}

// time_step_duration.f90:74-123 closing formula for on_going_time_step.
__device__ void tsd_close(const SimDev& s, SimDyn& d, double dtmin_cfl, int on_going) {
  double dtmin = kMaxPositive;
  double dt_vis = kMaxPositive;
  double dt;
  if (d.nag == 0) {
    dt = 0.0;
  } else {
    if (s.kin_visc > 1.0e-24) {
      dt_vis = s.vsc_coeff * s.squareh / (0.5 * s.kin_visc);
      dtmin = fmin(dtmin, dt_vis);
    }
    dtmin = fmin(dtmin, fmin(dtmin_cfl, dt_vis));
    if (s.dt_alfa_mon) {
      double visc_mon = s.alfa_mon * s.celerita * s.h / s.den0;
      double dt_mon = s.squareh / (0.5 * visc_mon);
      dtmin = fmin(dtmin, fmin(kMaxPositive, dt_mon));
    }
    if (on_going == 0) dt = dtmin;
    else dt = (1.0 - s.pesodt) * dtmin + s.pesodt * d.dt_average;
  }
  if (on_going == 0) d.dt_average = dt;
  else d.dt_average = (d.dt_average * (on_going - 1) + dt) / on_going;
  d.dt = dt;
}

// mode 0: IC.  time_step_loop.f90:173 evaluates dt with on_going_time_step
//         = -999, then the first iteration (time_step_loop.f90:182-185)
//         evaluates it again for step 1 from the same velocities.
// mode 1: end of a step: advance the simulation time and evaluate the dt of
//         the next iteration (its time_step_duration sees the velocities
//         this step left).
// Between steps the state keeps: step = completed steps, time = sum of their
// dt, dt = dt of the next step, dt_prev = dt of the last step.
// Sine of the tank forcing phase, written out so that host and device give
// the same bits: x is reduced by the nearest multiple of 2 pi into
// [-pi, pi], folded into [-pi/2, pi/2] by sin(r) = sin(+-pi - r), and the
// Taylor series of sin is summed to the r^23 term in nested form,
// r (1 - r^2/(2*3) (1 - r^2/(4*5) (...))), truncation below 1e-20 there.
// Every operation is a correctly rounded IEEE operation.
__device__ __forceinline__ double forcing_sin(double x) {
  const double two_pi = 6.283185307179586, pi = 3.141592653589793, half_pi = 1.5707963267948966;
  double k = rint(x / two_pi);
  double r = x - k * two_pi;
  if (r > half_pi) r = pi - r;
  else if (r < -half_pi) r = -pi - r;
  double r2 = r * r;
  double t = 1.0;
  for (int n = 22; n >= 2; n -= 2) t = 1.0 - r2 / (double)(n * (n + 1)) * t;
  return r * t;
}

__global__ void k_finalize(DevBatch b, int mode) {
  int sim = blockIdx.x * blockDim.x + threadIdx.x;
  if (sim >= b.nsims) return;
  const SimDev& s = b.sims[sim];
  SimDyn& d = b.dyn[sim];
  unsigned long long bits = d.dtmin_bits;
  double dtmin_cfl = (bits == 0x7FF0000000000000ull) ? kMaxPositive : __longlong_as_double((long long)bits);
  d.dtmin_bits = 0x7FF0000000000000ull;
  if (mode == 0) {
    d.dt_average = 0.0;
    tsd_close(s, d, dtmin_cfl, -999);
    double dt_ic = d.dt;
    tsd_close(s, d, dtmin_cfl, 1);
    d.dt_prev = dt_ic;
    d.step = 0;
    d.time = 0.0;
    d.frozen = 0;
  } else {
    if (d.frozen) return;
    d.time = d.time + d.dt;
    d.step = d.step + 1;
    double dt_cur = d.dt;
    tsd_close(s, d, dtmin_cfl, d.step + 1);
    d.dt_prev = dt_cur;
    if (d.t_end > 0.0 && d.time >= d.t_end) d.frozen = 1;
    // a simulation with a fatal status stops advancing; the others of its
    // batch go on (its segment, cells and boundary quota are its own)
    if (d.status != 0) d.frozen = 1;
  }
  d.dtvel = 0.5 * (d.dt + d.dt_prev);
  // body force of the next step, taken at that step's end time d.time + d.dt
  // (the simulation time when its momentum equation is evaluated): gravity,
  // plus the lateral forcing of a tank moving as x = A sin(w t) seen in the
  // tank frame, A w^2 sin(w t) along x (no reference counterpart; zero
  // amplitude leaves grav unchanged)
  d.geff[0] = s.forcing_aw2 != 0.0 ? s.grav[0] + s.forcing_aw2 * forcing_sin(s.forcing_w * (d.time + d.dt))
                                   : s.grav[0];
  d.geff[1] = s.grav[1];
  d.geff[2] = s.grav[2];
}

// sph_set_time_step: the next step's dt set from outside (the minimum over
// the slabs of a decomposed simulation, each of which closed its step with
// the minimum over its own particles).  With pesodt = 0 the closing's dt is
// that minimum itself, so the whole simulation's dt is the minimum of the
// slabs'; before the first step the IC's dt (dt_prev) is the same value.
// dtvel and the next step's body force follow from it as in k_finalize.
__global__ void k_set_dt(DevBatch b, double dt) {
  const int sim = blockIdx.x * blockDim.x + threadIdx.x;
  if (sim >= b.nsims) return;
  const SimDev& s = b.sims[sim];
  SimDyn& d = b.dyn[sim];
  d.dt = dt;
  if (d.step == 0) d.dt_prev = dt;
  d.dtvel = 0.5 * (d.dt + d.dt_prev);
  d.geff[0] = s.forcing_aw2 != 0.0 ? s.grav[0] + s.forcing_aw2 * forcing_sin(s.forcing_w * (d.time + d.dt))
                                   : s.grav[0];
}

// sph_set_clock: the clock of a resumed simulation (sim 0), with dtvel and
// the next step's body force as k_finalize leaves them.
__global__ void k_set_clock(DevBatch b, double time, int step, double dt, double dt_prev, double dt_average) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const SimDev& s = b.sims[0];
  SimDyn& d = b.dyn[0];
  d.time = time;
  d.step = step;
  d.dt = dt;
  d.dt_prev = dt_prev;
  d.dt_average = dt_average;
  d.dtvel = 0.5 * (d.dt + d.dt_prev);
  d.geff[0] = s.forcing_aw2 != 0.0 ? s.grav[0] + s.forcing_aw2 * forcing_sin(s.forcing_w * (d.time + d.dt))
                                   : s.grav[0];
}

// The laminar flags of a resumed simulation, from caller order.
__global__ void k_load_laminar(DevBatch b, const int* flags) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    P.L[p] = (uint8_t)(flags[(size_t)s.p_off + P.I[p] - 1] != 0);
  }
}

// sph_batch_cancel: a simulation still advancing stops from the next launch
// on, with status SPH_CANCELLED; one already frozen (finished or failed)
// keeps its status.
__global__ void k_cancel(DevBatch b, int sim) {
  if (threadIdx.x == 0 && sim < b.nsims && !b.dyn[sim].frozen) {
    atomicCAS(&b.dyn[sim].status, 0, SPH_CANCELLED);
    b.dyn[sim].frozen = 1;
  }
}

__global__ void k_sort_reset(DevBatch b) {
  int sim = blockIdx.x * blockDim.x + threadIdx.x;
  if (sim < b.nsims) b.dyn[sim].n_out = 0;
}

__global__ void k_bdt_reset(DevBatch b) {
  int sim = blockIdx.x * blockDim.x + threadIdx.x;
  if (sim < b.nsims) {
    b.dyn[sim].ncbf_max = 0;
    b.dyn[sim].bdt_sim_used = 0;
  }
  if (sim == 0) b.dyn[b.nsims].bdt_used = 0;
}

// ==========================================================================
// Global quantities (fluid_global_quantities.f90:59-72): FP64 sums over the
// fluid of mass, linear momentum, angular momentum about the origin
// (Vector_Product.f90 of coord and vel) and volume m / rho.  The reference
// sums sequentially in pg order; here each tile's particles are summed by a
// fixed shuffle tree and the tiles of a simulation in tile order, every
// addition compensated (a sum and its rounding error), so the result is the
// exact sum up to a few ulps and does not depend on the launch shape.
// ==========================================================================
struct CSum {
  double s, c;   // sum, accumulated rounding error
};

// TwoSum (Knuth) of the leading parts, the trailing parts added, then
// renormalised so |c| stays below an ulp of s.
__device__ __forceinline__ CSum csum_add(CSum a, CSum b) {
  const double s = a.s + b.s;
  const double bb = s - a.s;
  const double e = (a.s - (s - bb)) + (b.s - bb);
  const double c = (a.c + b.c) + e;
  const double t = s + c;
  return CSum{t, c - (t - s)};
}

__device__ __forceinline__ CSum csum_warp(CSum a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    CSum b{__shfl_down_sync(0xffffffffu, a.s, o), __shfl_down_sync(0xffffffffu, a.c, o)};
    a = csum_add(a, b);
  }
  return a;
}

constexpr int kGlobalQ = 8;

// Per-tile compensated partial sums: part[t][q] = (s, c).
__global__ void __launch_bounds__(kBlock) k_global_partials(DevBatch b, double2* part) {
  __shared__ SimDev s;
  __shared__ CSum ws[kBlock / 32][kGlobalQ];
  int cur = -1;
  const Particles& P = b.P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    const int p = tl.start + threadIdx.x;
    double q[kGlobalQ];
#pragma unroll
    for (int k = 0; k < kGlobalQ; ++k) q[k] = 0.0;
    if (threadIdx.x < tl.count && p < s.p_off + b.dyn[tl.sim].nag) {
      const double4 x = P.X[p];
      const double4 u = P.V[p];
      const double m = x.w;
      q[0] = m;
      q[1] = m * u.x;
      q[2] = m * u.y;
      q[3] = m * u.z;
      q[4] = m * (x.y * u.z - x.z * u.y);
      q[5] = m * (x.z * u.x - x.x * u.z);
      q[6] = m * (x.x * u.y - x.y * u.x);
      q[7] = m / P.RP[p].x;
    }
#pragma unroll
    for (int k = 0; k < kGlobalQ; ++k) {
      CSum a = csum_warp(CSum{q[k], 0.0});
      if (lane == 0) ws[warp][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < kGlobalQ) {
      CSum a = ws[0][threadIdx.x];
      for (int w = 1; w < kBlock / 32; ++w) a = csum_add(a, ws[w][threadIdx.x]);
      part[(size_t)t * kGlobalQ + threadIdx.x] = make_double2(a.s, a.c);
    }
    __syncthreads();
  }
}

// One warp per simulation: its tiles' partials in tile order (lane l takes
// tiles l, l + 32, ...), then the fixed shuffle tree.
__global__ void k_global_final(DevBatch b, const double2* __restrict__ part, double* out) {
  const int sim = blockIdx.x;
  const int lane = threadIdx.x;
  const int t0 = b.sims[sim].p_off / kBlock;
  const int t1 = t0 + (b.sims[sim].cap + kBlock - 1) / kBlock;
  for (int k = 0; k < kGlobalQ; ++k) {
    CSum a{0.0, 0.0};
    for (int t = t0 + lane; t < t1; t += 32) {
      const double2 v = part[(size_t)t * kGlobalQ + k];
      a = csum_add(a, CSum{v.x, v.y});
    }
    a = csum_warp(a);
    if (lane == 0) out[(size_t)sim * kGlobalQ + k] = a.s + a.c;
  }
}

// ==========================================================================
// Caller-order transfer and verification dumps
// ==========================================================================
__global__ void k_init_from_caller(DevBatch b, const double* x, const double* v, const double* rho, const double* p,
                                   const double* m) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int q = tl.start + threadIdx.x;           // caller order slot
    int i = q - s.p_off;                       // caller index - 1
    if (i < b.dyn[tl.sim].nag) {
      P.X2[q] = make_double4(x[3 * (size_t)q], x[3 * (size_t)q + 1], x[3 * (size_t)q + 2], m[q]);
      P.V2[q] = make_double4(v[3 * (size_t)q], v[3 * (size_t)q + 1], v[3 * (size_t)q + 2], rho[q]);
      P.P2[q] = p[q];
      P.I2[q] = i + 1;
    } else {
      P.X2[q] = make_double4(0, 0, 0, 0);
      P.V2[q] = make_double4(0, 0, 0, 1.0);
      P.P2[q] = 0.0;
      P.I2[q] = 0;
    }
    P.L2[q] = 0;
  }
}

// k_init_from_caller in two halves, for an upload whose positions and
// masses arrive first: the positions half also marks each slot's caller
// index (0 = empty), and the rest half fills a slot's velocity, density and
// pressure where that mark is set.  The rest half does not read the particle
// count, which the removal pass of the concurrent sort may be lowering.
__global__ void k_init_positions(DevBatch b, const double* x, const double* m) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    if (threadIdx.x >= tl.count) continue;
    int q = tl.start + threadIdx.x;
    int i = q - s.p_off;
    if (i < b.dyn[tl.sim].nag) {
      P.X2[q] = make_double4(x[3 * (size_t)q], x[3 * (size_t)q + 1], x[3 * (size_t)q + 2], m[q]);
      P.I2[q] = i + 1;
    } else {
      P.X2[q] = make_double4(0, 0, 0, 0);
      P.I2[q] = 0;
    }
    P.L2[q] = 0;
  }
}

__global__ void k_init_rest(DevBatch b, const double* v, const double* rho, const double* p) {
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    if (threadIdx.x >= tl.count) continue;
    int q = tl.start + threadIdx.x;
    if (P.I2[q] != 0) {
      P.V2[q] = make_double4(v[3 * (size_t)q], v[3 * (size_t)q + 1], v[3 * (size_t)q + 2], rho[q]);
      P.P2[q] = p[q];
    } else {
      P.V2[q] = make_double4(0, 0, 0, 1.0);
      P.P2[q] = 0.0;
    }
  }
}

__global__ void k_to_caller(DevBatch b, double* x, double* v, double* rho, double* p, double* m, double* acc,
                            double* dden) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int q = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || q >= s.p_off + b.dyn[tl.sim].nag) continue;
    size_t o = (size_t)s.p_off + P.I[q] - 1;
    double4 xx = P.X[q];
    double4 vv = P.V[q];
    double2 rp = P.RP[q];
    if (x) { x[3 * o] = xx.x; x[3 * o + 1] = xx.y; x[3 * o + 2] = xx.z; }
    if (v) { v[3 * o] = vv.x; v[3 * o + 1] = vv.y; v[3 * o + 2] = vv.z; }
    if (rho) rho[o] = rp.x;
    if (p) p[o] = rp.y;
    if (m) m[o] = xx.w;
    if (acc) { double4 a = P.ACC[q]; acc[3 * o] = a.x; acc[3 * o + 1] = a.y; acc[3 * o + 2] = a.z; }
    if (dden) dden[o] = P.DDEN[q];
  }
}

// Positions, velocities and masses of a fused step's record (X2, V2, I2 in
// the last sort's slot order, written by the momentum pass and final from
// then on) to caller order, before the step's own sort has run.  Slots are
// those below the particle count; the sort's removal pass may lower that
// count concurrently, in which case the caller redoes this copy from the
// sorted state (the removal renumbers particles).
__global__ void k_scratch_to_caller(DevBatch b, double* x, double* v, double* m) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int q = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || q >= s.p_off + b.dyn[tl.sim].nag) continue;
    const int id = P.I2[q];
    if (id <= 0) continue;
    const size_t o = (size_t)s.p_off + id - 1;
    const double4 xx = P.X2[q];
    const double4 vv = P.V2[q];
    x[3 * o] = xx.x; x[3 * o + 1] = xx.y; x[3 * o + 2] = xx.z;
    v[3 * o] = vv.x; v[3 * o + 1] = vv.y; v[3 * o + 2] = vv.z;
    m[o] = xx.w;
  }
}

template <int DIM>
__global__ void k_dump_neighbours(DevBatch b, int nmaxj, int* counts, int* lists) {
  // the stored lists the pair passes read, in caller indices, with the
  // particle itself put back where the reference's visiting order has it
  // (the lists leave it out): before the first entry past its own slot in
  // its own column (the centre run).  It was accepted unless the NMAXPARTJ
  // cap cut the list before it, in which case cnt reached the cap.
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  constexpr unsigned kCentre = (DIM == 3) ? 4u : 1u;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    size_t row = (size_t)s.p_off + P.I[p] - 1;
    const int cnt = b.ncount[p];
    const int* base = reinterpret_cast<const int*>(reinterpret_cast<const int4*>(b.nlist) + list_base4(p, b.list_cap4));
    bool self = cnt < s.nmaxpartj;
    int n = 0;
    for (int k = 0; k < cnt; ++k) {
      const unsigned e = (unsigned)base[(size_t)(k >> 2) * 128 + (k & 3)];
      const unsigned run = e >> kSlotBits;
      const int q = (int)(e & kSlotMask);
      if (self && (run > kCentre || (run == kCentre && q > p))) {
        if (n < nmaxj) lists[row * nmaxj + n] = P.I[p];
        n++;
        self = false;
      }
      if (n < nmaxj) lists[row * nmaxj + n] = P.I[q];
      n++;
    }
    if (self) {
      if (n < nmaxj) lists[row * nmaxj + n] = P.I[p];
      n++;
    }
    counts[row] = n;
  }
}

__global__ void k_dump_boundary(DevBatch b, int max_per, int* ncb, int* clob, double* vals) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    size_t row = (size_t)s.p_off + P.I[p] - 1;
    int n = P.bdt_count[p];
    ncb[row] = n;
    for (int k = 0; k < n && k < max_per; ++k) {
      const BdtEntry& e = P.bdt[P.bdt_start[p] + k];
      clob[row * max_per + k] = e.clobonum;
      double* d = vals + (row * max_per + k) * 20;
      for (int q = 0; q < 3; ++q) d[q] = e.loc[q];
      for (int q = 0; q < 8; ++q) d[3 + q] = e.bi[q];
      // IntGiWrRdV(3,3) column-major
      for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r) d[11 + 3 * c + r] = e.ig[3 * r + c];
    }
  }
}

// B_ren_gradp / B_ren_divu by caller index, B(i,j) at [9 row + 3 i + j].
__global__ void k_dump_renormalisation(DevBatch b, double* bg, double* bd) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    size_t row = (size_t)s.p_off + P.I[p] - 1;
    for (int k = 0; k < 9; ++k) {
      if (bg && P.BG) bg[9 * row + k] = P.BG[(size_t)k * P.total_slots + p];
      if (bd && P.BD) bd[9 * row + k] = P.BD[(size_t)k * P.total_slots + p];
    }
  }
}

__global__ void k_dump_cella(DevBatch b, int* cella) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    double4 xi = P.X[p];
    int i, j, k;
    int c = 0;
    if (particle_cell(s, xi.x, xi.y, xi.z, i, j, k)) c = ((k - 1) * s.ncd[1] + (j - 1)) * s.ncd[0] + i;
    cella[(size_t)s.p_off + P.I[p] - 1] = c;
  }
}

// pg%laminar_flag (inter_EqMoto.f90:269-283) of the last momentum pass, in
// caller order.
__global__ void k_dump_laminar(DevBatch b, int* flags) {
  __shared__ SimDev s;
  int cur = -1;
  const Particles& P = b.P;
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    Tile tl = b.tiles[t];
    load_sim(s, b.sims, tl.sim, cur);
    int p = tl.start + threadIdx.x;
    if (threadIdx.x >= tl.count || p >= s.p_off + b.dyn[tl.sim].nag) continue;
    flags[(size_t)s.p_off + P.I[p] - 1] = P.L[p];
  }
}

// FP64 fused multiply-add throughput probe (8 independent chains per thread).
__global__ void __launch_bounds__(256) k_fp64_probe(double* sink, int iters) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double m = 0.999999999, c = 1e-12;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
    a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
  }
  double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 12345.0) sink[blockIdx.x] = r;
}

// FP32 fused multiply-add throughput probe.
__global__ void __launch_bounds__(256) k_fp32_probe(float* sink, int iters) {
  float a0 = threadIdx.x * 1e-6f, a1 = a0 + 1e-6f, a2 = a0 + 2e-6f, a3 = a0 + 3e-6f;
  float a4 = a0 + 4e-6f, a5 = a0 + 5e-6f, a6 = a0 + 6e-6f, a7 = a0 + 7e-6f;
  const float m = 0.9999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
    a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
    a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
  }
  float r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 12345.0f) sink[blockIdx.x] = r;
}

double launch_fp32_probe(float* sink, int blocks, cudaStream_t st) {
  const int iters = 8192;
  k_fp32_probe<<<blocks, 256, 0, st>>>(sink, iters);
  return 2.0 * 8.0 * iters * 256.0 * blocks;
}

double launch_fp64_probe(double* sink, int blocks, cudaStream_t st) {
  const int iters = 4096;
  k_fp64_probe<<<blocks, 256, 0, st>>>(sink, iters);
  return 2.0 * 8.0 * iters * 256.0 * blocks;
}

// Self-check of div_rn against the IEEE division a / b on generated
// operands (SplitMix64 of the seed and the operand index).  Five kinds, by
// index mod 5: random signs, significands and exponents in [-64, 63];
// divisors whose significands are within 255 units of all ones; quotients
// within a few units of 2^-106 relative of a rounding midpoint of a random
// quotient (a = RN(b q + b ulp(q)/2)); a zero dividend of either sign; and
// the ranges of the kernels' operands (1e-6 to 1e3 over 1e-3 to 2e3).
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double compose_double(unsigned long long frac, int exp, unsigned sign) {
  const unsigned long long bits = ((unsigned long long)(sign & 1u) << 63) |
                                  ((unsigned long long)(exp + 1023) << 52) | (frac & ((1ull << 52) - 1));
  return __longlong_as_double((long long)bits);
}

// bad[0] counts mismatches, bad[1] flags that first[] holds one's operands.
__global__ void __launch_bounds__(256) k_check_division(unsigned long long n, unsigned long long seed,
                                                        unsigned long long* bad, double* first) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long nbad = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long u1 = splitmix64(seed ^ (2 * i)), u2 = splitmix64(seed ^ (2 * i + 1));
    const int e1 = (int)((u1 >> 52) & 127) - 64, e2 = (int)((u2 >> 52) & 127) - 64;
    double a, b;
    switch ((int)(i % 5)) {
      case 0:
        a = compose_double(u1, e1, (unsigned)(u1 >> 63));
        b = compose_double(u2, e2, (unsigned)(u2 >> 63));
        break;
      case 1:
        a = compose_double(u1, e1, (unsigned)(u1 >> 63));
        b = compose_double(((1ull << 52) - 1) - (u2 & 255), e2 & 15, (unsigned)(u2 >> 63));
        break;
      case 2: {
        const double q = compose_double(u1, e1 & 31, 0);
        const double half_ulp = compose_double(0, (e1 & 31) - 53, 0);
        b = compose_double(u2, e2 & 31, (unsigned)(u2 >> 63));
        a = __fma_rn(b, half_ulp, __dmul_rn(b, q));
        break;
      }
      case 3:
        a = (u1 & 1) ? -0.0 : 0.0;
        b = compose_double(u2, e2, (unsigned)(u2 >> 63));
        break;
      default:
        a = compose_double(u1, (int)((u1 >> 52) % 30) - 20, (unsigned)(u1 >> 63));
        b = compose_double(u2, (int)((u2 >> 52) % 21) - 10, 0);
        break;
    }
    const double ref = a / b;
    const double got = div_rn(a, b, __drcp_rn(b));
    if (__double_as_longlong(ref) != __double_as_longlong(got)) {
      ++nbad;
      if (atomicCAS(bad + 1, 0ull, 1ull) == 0ull) {   // the first mismatch found keeps its operands
        first[0] = a;
        first[1] = b;
      }
    }
  }
  if (nbad) atomicAdd(bad, nbad);
}

void launch_check_division(unsigned long long n, unsigned long long seed, unsigned long long* bad, double* first,
                           int blocks, cudaStream_t st) {
  k_check_division<<<blocks, 256, 0, st>>>(n, seed, bad, first);
}

// ==========================================================================
// launch wrappers
// ==========================================================================
static inline int blocks_for(const DevBatch& b) { return b.ntiles < b.grid_blocks ? b.ntiles : b.grid_blocks; }
static inline int blocks_for(const DevBatch& b, int cls) {
  int g = b.grid[cls] > 0 ? b.grid[cls] : b.grid_blocks;
  return b.ntiles < g ? b.ntiles : g;
}

void launch_stage(const DevBatch& b, cudaStream_t st) { k_stage<<<blocks_for(b), kBlock, 0, st>>>(b); }

void launch_bin(const DevBatch& b, KeyKind kind, cudaStream_t st) {
  if (kind == KeyKind::Sort) k_bin<KeyKind::Sort><<<blocks_for(b), kBlock, 0, st>>>(b);
  else k_bin<KeyKind::Reference><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_removal(const DevBatch& b, cudaStream_t st) { k_removal<<<b.nsims, 32, 0, st>>>(b); }

void launch_scan(const DevBatch& b, int* cell_start, cudaStream_t st) {
  int n = b.P.total_cells;
  int nb = (n + kScanChunk - 1) / kScanChunk;
  k_scan1<<<nb, kScanThreads, 0, st>>>(b.P.cell_count, n, b.scan_block_sums);
  k_scan2<<<1, kScanThreads, 0, st>>>(b.scan_block_sums, nb, cell_start, n);
  k_scan3<<<nb, kScanThreads, 0, st>>>(b.P.cell_count, n, b.scan_block_sums, cell_start);
}

void launch_cancel(const DevBatch& b, int sim, cudaStream_t st) { k_cancel<<<1, 32, 0, st>>>(b, sim); }

void launch_load_laminar(const DevBatch& b, const int* laminar, cudaStream_t st) {
  k_load_laminar<<<blocks_for(b), kBlock, 0, st>>>(b, laminar);
}
void launch_set_clock(const DevBatch& b, double time, int step, double dt, double dt_prev, double dt_average,
                      const int* laminar, cudaStream_t st) {
  k_set_clock<<<1, 32, 0, st>>>(b, time, step, dt, dt_prev, dt_average);
  if (laminar) launch_load_laminar(b, laminar, st);
}
void launch_set_dt(const DevBatch& b, double dt, cudaStream_t st) {
  k_set_dt<<<(b.nsims + 127) / 128, 128, 0, st>>>(b, dt);
}

void launch_sort_reset(const DevBatch& b, cudaStream_t st) {
  k_sort_reset<<<(b.nsims + 127) / 128, 128, 0, st>>>(b);
}

void upload_bit2d(const double* tab, cudaStream_t st) {
  cudaMemcpyToSymbolAsync(c_bit2d, tab, sizeof(double) * 22 * 6, 0, cudaMemcpyHostToDevice, st);
}

void launch_place(const DevBatch& b, cudaStream_t st) {
  k_place<<<blocks_for(b), kBlock, 0, st>>>(b, b.P.cell_start, 1);
}

void launch_rank_permute(const DevBatch& b, cudaStream_t st) {
  k_rank_permute<kPermuteAll><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_rank_permute_positions(const DevBatch& b, cudaStream_t st) {
  k_rank_permute<kPermutePositions><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_rank_permute_rest(const DevBatch& b, cudaStream_t st) {
  k_rank_permute<kPermuteRest><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_rank_reference(const DevBatch& b, const int* cell_start_ref, int* npartord, cudaStream_t st) {
  k_place<<<blocks_for(b), kBlock, 0, st>>>(b, cell_start_ref, 0);
  k_rank_reference<<<blocks_for(b), kBlock, 0, st>>>(b, cell_start_ref, npartord);
}

void launch_boundary(const DevBatch& b, cudaStream_t st) {
  k_bdt_reset<<<(b.nsims + 127) / 128, 128, 0, st>>>(b);
  if (b.dim == 3) {
    k_boundary3d<<<blocks_for(b, kGridBoundary), kBlock, 0, st>>>(b);
    k_boundary3d_integrals<<<b.grid[kGridIntegrals] > 0 ? b.grid[kGridIntegrals] : b.grid_blocks * 2, 128, 0, st>>>(b);
  } else {
    k_boundary2d<<<blocks_for(b, kGridBoundary), kBlock, 0, st>>>(b);
  }
}

// 2D with C1_BE: the frontier terms and inversion of the matrices (their
// renormalisation is the identity in 2D, see k_c1_frontier_2d)
static void c1_frontier_2d(const DevBatch& b, bool gradp_only, cudaStream_t st) {
  if (b.dim != 2 || !b.c1) return;
  if (gradp_only) k_c1_frontier_2d<true><<<blocks_for(b), kBlock, 0, st>>>(b);
  else k_c1_frontier_2d<false><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_momentum(const DevBatch& b, bool fused, cudaStream_t st) {
  int g = blocks_for(b, kGridMomentum);
  c1_frontier_2d(b, true, st);
  if (b.dim == 3 && b.c1) {
    if (fused) k_momentum<3, true, true><<<g, kBlock, 0, st>>>(b);
    else k_momentum<3, false, true><<<g, kBlock, 0, st>>>(b);
  } else if (b.dim == 3) {
    if (b.mom_batch) {
      if (fused) k_momentum<3, true, false, true><<<g, kBlock, 0, st>>>(b);
      else k_momentum<3, false, false, true><<<g, kBlock, 0, st>>>(b);
    } else {
      if (fused) k_momentum<3, true><<<g, kBlock, 0, st>>>(b);
      else k_momentum<3, false><<<g, kBlock, 0, st>>>(b);
    }
  } else {
    if (b.mom_batch) {
      if (fused) k_momentum<2, true, false, true><<<g, kBlock, 0, st>>>(b);
      else k_momentum<2, false, false, true><<<g, kBlock, 0, st>>>(b);
    } else {
      if (fused) k_momentum<2, true><<<g, kBlock, 0, st>>>(b);
      else k_momentum<2, false><<<g, kBlock, 0, st>>>(b);
    }
  }
}

void launch_neighbour_lists(const DevBatch& b, cudaStream_t st) {
  int g = blocks_for(b, kGridLists);
  if (b.dim == 3) k_neighbour_lists<3><<<g, kBlock, 0, st>>>(b);
  else k_neighbour_lists<2><<<g, kBlock, 0, st>>>(b);
}

void launch_renormalisation(const DevBatch& b, cudaStream_t st) {
  if (!b.c1) return;
  if (b.dim == 3) k_renormalisation<3><<<blocks_for(b, kGridLists), kBlock, 0, st>>>(b);
  else k_renormalisation<2><<<blocks_for(b, kGridLists), kBlock, 0, st>>>(b);
}

void launch_momentum_f32(const DevBatch& b, bool fused, cudaStream_t st) {
  int g = blocks_for(b, kGridMomentum);
  int gf = blocks_for(b);
  c1_frontier_2d(b, true, st);
  const int f = fused ? 1 : 0;
  if (b.dim == 3 && b.c1) {
    k_momentum_f32<3, true><<<g, kBlock, 0, st>>>(b, f);
    if (fused) k_momentum_f32_finish<3, true, true><<<gf, kBlock, 0, st>>>(b);
    else k_momentum_f32_finish<3, false, true><<<gf, kBlock, 0, st>>>(b);
  } else if (b.dim == 3) {
    if (b.mom_batch == 2) k_momentum_f32<3, false, true, true><<<g, kBlock, 0, st>>>(b, f);
    else if (b.mom_batch) k_momentum_f32<3, false, true><<<g, kBlock, 0, st>>>(b, f);
    else k_momentum_f32<3><<<g, kBlock, 0, st>>>(b, f);
    if (fused) k_momentum_f32_finish<3, true><<<gf, kBlock, 0, st>>>(b);
    else k_momentum_f32_finish<3, false><<<gf, kBlock, 0, st>>>(b);
  } else {
    if (b.mom_batch == 2) k_momentum_f32<2, false, true, true><<<g, kBlock, 0, st>>>(b, f);
    else if (b.mom_batch) k_momentum_f32<2, false, true><<<g, kBlock, 0, st>>>(b, f);
    else k_momentum_f32<2><<<g, kBlock, 0, st>>>(b, f);
    if (fused) k_momentum_f32_finish<2, true><<<gf, kBlock, 0, st>>>(b);
    else k_momentum_f32_finish<2, false><<<gf, kBlock, 0, st>>>(b);
  }
}

void launch_continuity_f32_pairs(const DevBatch& b, cudaStream_t st) {
  int g = blocks_for(b, kGridContinuity);
  if (b.dim == 3 && b.c1_divu) k_continuity_f32<3, true><<<g, kBlock, 0, st>>>(b);
  else if (b.dim == 3 && b.con_batch == 2) k_continuity_f32<3, false, true, true><<<g, kBlock, 0, st>>>(b);
  else if (b.dim == 3 && b.con_batch) k_continuity_f32<3, false, true><<<g, kBlock, 0, st>>>(b);
  else if (b.dim == 3) k_continuity_f32<3><<<g, kBlock, 0, st>>>(b);
  else if (b.con_batch == 2) k_continuity_f32<2, false, true, true><<<g, kBlock, 0, st>>>(b);
  else if (b.con_batch) k_continuity_f32<2, false, true><<<g, kBlock, 0, st>>>(b);
  else k_continuity_f32<2><<<g, kBlock, 0, st>>>(b);
}

void launch_continuity_f32_finish(const DevBatch& b, bool fused, cudaStream_t st) {
  int g = blocks_for(b);
  c1_frontier_2d(b, false, st);
  if (b.dim == 3 && b.c1) {
    if (fused) k_continuity_f32_finish<3, true, true><<<g, kBlock, 0, st>>>(b);
    else k_continuity_f32_finish<3, false, true><<<g, kBlock, 0, st>>>(b);
  } else if (b.dim == 3) {
    if (fused) k_continuity_f32_finish<3, true><<<g, kBlock, 0, st>>>(b);
    else k_continuity_f32_finish<3, false><<<g, kBlock, 0, st>>>(b);
  } else {
    if (fused) k_continuity_f32_finish<2, true><<<g, kBlock, 0, st>>>(b);
    else k_continuity_f32_finish<2, false><<<g, kBlock, 0, st>>>(b);
  }
}

void launch_continuity_f32(const DevBatch& b, bool fused, cudaStream_t st) {
  launch_continuity_f32_pairs(b, st);
  launch_continuity_f32_finish(b, fused, st);
}

void launch_refresh_f32(const DevBatch& b, cudaStream_t st) { k_refresh_f32<<<blocks_for(b), kBlock, 0, st>>>(b); }

void launch_continuity(const DevBatch& b, bool fused, cudaStream_t st) {
  int g = blocks_for(b, kGridContinuity);
  c1_frontier_2d(b, false, st);
  if (b.dim == 3 && b.c1) {
    if (fused) k_continuity<3, true, true><<<g, kBlock, 0, st>>>(b);
    else k_continuity<3, false, true><<<g, kBlock, 0, st>>>(b);
  } else if (b.dim == 3) {
    if (b.con_batch) {
      if (fused) k_continuity<3, true, false, true><<<g, kBlock, 0, st>>>(b);
      else k_continuity<3, false, false, true><<<g, kBlock, 0, st>>>(b);
    } else {
      if (fused) k_continuity<3, true><<<g, kBlock, 0, st>>>(b);
      else k_continuity<3, false><<<g, kBlock, 0, st>>>(b);
    }
  } else {
    if (b.con_batch) {
      if (fused) k_continuity<2, true, false, true><<<g, kBlock, 0, st>>>(b);
      else k_continuity<2, false, false, true><<<g, kBlock, 0, st>>>(b);
    } else {
      if (fused) k_continuity<2, true><<<g, kBlock, 0, st>>>(b);
      else k_continuity<2, false><<<g, kBlock, 0, st>>>(b);
    }
  }
}

void launch_leapfrog_momentum(const DevBatch& b, cudaStream_t st) {
  k_leapfrog_momentum<<<blocks_for(b), kBlock, 0, st>>>(b);
}
void launch_leapfrog_trajectories(const DevBatch& b, cudaStream_t st) {
  k_leapfrog_trajectories<<<blocks_for(b), kBlock, 0, st>>>(b);
}
void launch_leapfrog_continuity(const DevBatch& b, cudaStream_t st) {
  k_leapfrog_continuity<<<blocks_for(b), kBlock, 0, st>>>(b);
}
void launch_eos(const DevBatch& b, cudaStream_t st) { k_eos<<<blocks_for(b), kBlock, 0, st>>>(b); }

void launch_velocity_smoothing(const DevBatch& b, bool fused, bool fp32c, cudaStream_t st) {
  const double4* vel = fused ? b.P.V2 : b.P.V;
  if (fp32c) {
    if (b.dim == 3) k_velocity_smoothing_f32<3><<<blocks_for(b), kBlock, 0, st>>>(b, vel);
    else k_velocity_smoothing_f32<2><<<blocks_for(b), kBlock, 0, st>>>(b, vel);
  } else {
    if (b.dim == 3) k_velocity_smoothing<3><<<blocks_for(b), kBlock, 0, st>>>(b, vel);
    else k_velocity_smoothing<2><<<blocks_for(b), kBlock, 0, st>>>(b, vel);
  }
  if (fused) k_velocity_smoothing_apply<true><<<blocks_for(b), kBlock, 0, st>>>(b);
  else k_velocity_smoothing_apply<false><<<blocks_for(b), kBlock, 0, st>>>(b);
}

void launch_pressure_smoothing(const DevBatch& b, bool fp32c, cudaStream_t st) {
  const bool refresh_f32 = fp32c;
  if (fp32c) {
    if (b.dim == 3) k_pressure_smoothing_f32<3><<<blocks_for(b), kBlock, 0, st>>>(b);
    else k_pressure_smoothing_f32<2><<<blocks_for(b), kBlock, 0, st>>>(b);
  } else {
    if (b.dim == 3) k_pressure_smoothing<3><<<blocks_for(b), kBlock, 0, st>>>(b);
    else k_pressure_smoothing<2><<<blocks_for(b), kBlock, 0, st>>>(b);
  }
  k_pressure_smoothing_apply<<<blocks_for(b), kBlock, 0, st>>>(b, refresh_f32 ? 1 : 0);
}
void launch_dt_reduce(const DevBatch& b, cudaStream_t st) { k_dt_reduce<<<blocks_for(b), kBlock, 0, st>>>(b); }
void launch_finalize(const DevBatch& b, int mode, cudaStream_t st) {
  k_finalize<<<(b.nsims + 127) / 128, 128, 0, st>>>(b, mode);
}

void launch_init_from_caller(const DevBatch& b, const double* x, const double* v, const double* rho,
                             const double* p, const double* m, cudaStream_t st) {
  k_init_from_caller<<<blocks_for(b), kBlock, 0, st>>>(b, x, v, rho, p, m);
}
void launch_scratch_to_caller(const DevBatch& b, double* x, double* v, double* m, cudaStream_t st) {
  k_scratch_to_caller<<<blocks_for(b), kBlock, 0, st>>>(b, x, v, m);
}
void launch_init_positions(const DevBatch& b, const double* x, const double* m, cudaStream_t st) {
  k_init_positions<<<blocks_for(b), kBlock, 0, st>>>(b, x, m);
}
void launch_init_rest(const DevBatch& b, const double* v, const double* rho, const double* p, cudaStream_t st) {
  k_init_rest<<<blocks_for(b), kBlock, 0, st>>>(b, v, rho, p);
}
void launch_to_caller(const DevBatch& b, double* x, double* v, double* rho, double* p, double* m, double* acc,
                      double* dden, cudaStream_t st) {
  k_to_caller<<<blocks_for(b), kBlock, 0, st>>>(b, x, v, rho, p, m, acc, dden);
}
void launch_dump_neighbours(const DevBatch& b, int nmaxj, int* counts, int* lists, cudaStream_t st) {
  if (b.dim == 3) k_dump_neighbours<3><<<blocks_for(b), kBlock, 0, st>>>(b, nmaxj, counts, lists);
  else k_dump_neighbours<2><<<blocks_for(b), kBlock, 0, st>>>(b, nmaxj, counts, lists);
}
void launch_dump_boundary(const DevBatch& b, int max_per, int* ncb, int* clob, double* vals, cudaStream_t st) {
  k_dump_boundary<<<blocks_for(b), kBlock, 0, st>>>(b, max_per, ncb, clob, vals);
}
void launch_dump_renormalisation(const DevBatch& b, double* bg, double* bd, cudaStream_t st) {
  k_dump_renormalisation<<<blocks_for(b), kBlock, 0, st>>>(b, bg, bd);
}
void launch_global_quantities(const DevBatch& b, double2* part, double* out, cudaStream_t st) {
  k_global_partials<<<blocks_for(b), kBlock, 0, st>>>(b, part);
  k_global_final<<<b.nsims, 32, 0, st>>>(b, part, out);
}

void launch_dump_cella(const DevBatch& b, int* cella, cudaStream_t st) {
  k_dump_cella<<<blocks_for(b), kBlock, 0, st>>>(b, cella);
}

void launch_dump_laminar(const DevBatch& b, int* flags, cudaStream_t st) {
  k_dump_laminar<<<blocks_for(b), kBlock, 0, st>>>(b, flags);
}

}  // namespace sph
