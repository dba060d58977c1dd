// C ABI of the library (include/sphera_b200.h) and its host-side runtime:
// IC-time geometry and integral tables, device memory, the per-step launch
// sequence and its CUDA graph.
//
// Host arithmetic that feeds the kernels (grid, face frames, tables) is
// compiled with -ffp-contract=off and written in the reference's evaluation
// order, so the device sees the same constants the reference computes.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <algorithm>
#include <new>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sphera_b200.h"
#include "sph_internal.cuh"
#include "sph_launch.h"

// NVTX ranges around the entry points, named after the reference routines
// they stand in for, so a profiler's timeline reads like time_step_loop.f90
// (header-only; without a profiler attached a range costs a branch).
namespace {
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

namespace sph {

// BoundIntegralTab2D, SA_SPH_module.f90:29-54.  The DATA statement's values
// are default-REAL (single precision) literals, so the reference's double
// array holds their float roundings; kept here as float literals.
static const float kBit2dLiterals[22][6] = {
    {-9.900000E-02f, 6.916001E-01f, 5.671769E-01f, 1.614238E+00f, 7.329450E-01f, 8.813822E-01f},
    {1.000000E-03f, 6.820633E-01f, 4.993001E-01f, 1.426603E+00f, 7.142813E-01f, 7.123606E-01f},
    {1.010000E-01f, 6.725266E-01f, 4.314232E-01f, 1.238968E+00f, 6.956176E-01f, 5.433391E-01f},
    {2.010000E-01f, 6.452481E-01f, 3.653947E-01f, 1.057834E+00f, 6.492812E-01f, 4.085521E-01f},
    {3.010000E-01f, 6.025034E-01f, 3.028878E-01f, 8.871524E-01f, 5.851007E-01f, 3.020341E-01f},
    {4.010000E-01f, 5.473293E-01f, 2.453079E-01f, 7.296175E-01f, 5.106232E-01f, 2.189841E-01f},
    {5.010000E-01f, 4.832434E-01f, 1.937172E-01f, 5.872117E-01f, 4.319031E-01f, 1.553082E-01f},
    {6.010000E-01f, 4.139976E-01f, 1.488267E-01f, 4.612826E-01f, 3.538107E-01f, 1.074685E-01f},
    {7.010000E-01f, 3.434138E-01f, 1.109601E-01f, 3.526284E-01f, 2.802530E-01f, 7.237218E-02f},
    {8.010000E-01f, 2.751568E-01f, 8.006434E-02f, 2.615428E-01f, 2.142205E-01f, 4.732315E-02f},
    {9.010000E-01f, 2.125249E-01f, 5.573915E-02f, 1.877770E-01f, 1.577964E-01f, 2.998003E-02f},
    {1.001000E+00f, 1.581202E-01f, 3.728314E-02f, 1.304301E-01f, 1.120873E-01f, 1.834320E-02f},
    {1.101000E+00f, 1.131765E-01f, 2.379696E-02f, 8.756287E-02f, 7.679627E-02f, 1.076657E-02f},
    {1.201000E+00f, 7.737532E-02f, 1.434262E-02f, 5.638309E-02f, 5.038764E-02f, 5.995379E-03f},
    {1.301000E+00f, 4.995510E-02f, 8.042085E-03f, 3.441001E-02f, 3.129118E-02f, 3.118804E-03f},
    {1.401000E+00f, 2.994721E-02f, 4.104289E-03f, 1.956203E-02f, 1.807987E-02f, 1.482120E-03f},
    {1.501000E+00f, 1.623613E-02f, 1.842642E-03f, 1.008625E-02f, 9.464607E-03f, 6.216584E-04f},
    {1.601000E+00f, 7.615461E-03f, 6.873181E-04f, 4.510624E-03f, 4.293336E-03f, 2.172841E-04f},
    {1.701000E+00f, 2.842820E-03f, 1.913104E-04f, 1.609094E-03f, 1.552266E-03f, 5.682598E-05f},
    {1.801000E+00f, 6.998383E-04f, 3.120105E-05f, 3.793334E-04f, 3.706037E-04f, 8.729655E-06f},
    {1.901000E+00f, 6.214235E-05f, 1.372448E-06f, 3.231651E-05f, 3.195398E-05f, 3.625237E-07f},
    {2.001000E+00f, 0.000000E+00f, 0.000000E+00f, 0.000000E+00f, 0.000000E+00f, 0.000000E+00f}};

namespace {

constexpr double kPi = 3.14159265358979e0;   // PIGRECO, Static_allocation_module.f90:50

// One simulation as prepared on the host.
struct HostSim {
  SphParams prm{};
  SimDev dev{};
  std::vector<FaceDev> faces;
  std::vector<SideDev> sides;
  std::vector<EdgeDev> edges;          // convex edges (3D)
  std::vector<double> bit;             // 256 x 7
  std::vector<int> cf_count, cf_start, cf_list;
  std::vector<uint8_t> near;
  int cap = 0;
};

struct FaceGeo {   // host copy of a face for the cell-intersection test
  int nodes;
  double GX[6][3];
  double T[3][3];
  int zone;
};

// JdWsRn.f90 (beta-spline kernel, n = 1..3)
double jdwsrn(double ro, int n) {
  const double KS3D = 0.31830989;
  double ro2 = ro * ro, ro3 = ro2 * ro, ro4 = ro2 * ro2, ro5 = ro4 * ro;
  double J = 0.0;
  if (n == 1) {
    if (ro >= 0.0 && ro < 1.0) J = -0.75 + (1.0 - 0.5625 * ro) * ro3;
    else if (ro >= 1.0 && ro < 2.0) J = -1.0 + (1.5 - 1.0 * ro + 0.1875 * ro2) * ro2;
  } else if (n == 2) {
    if (ro >= 0.0 && ro < 1.0) J = -0.7 + (0.75 - 0.45 * ro) * ro4;
    else if (ro >= 1.0 && ro < 2.0) J = -0.8 + (1.0 - 0.75 * ro + 0.15 * ro2) * ro3;
  } else if (n == 3) {
    if (ro >= 0.0 && ro < 1.0) J = -0.75 + (0.6 - 0.375 * ro) * ro5;
    else if (ro >= 1.0 && ro < 2.0) J = -0.8 + (0.75 - 0.6 * ro + 0.125 * ro2) * ro4;
  }
  return J * KS3D;
}

// IWro2dro.f90:60-74
double iwro2dro(double ro) {
  const double a1 = 0.333333333333333, a2 = 0.3, a3 = 0.125, a4 = 0.25;
  const double b1 = 0.0625, b2 = 0.025, b3 = 4.16666666666667e-03;
  const double kc = 1.0 / kPi;
  if (ro >= 0.0 && ro < 1.0) {
    double ro2 = ro * ro, ro3 = ro2 * ro;
    double I1 = (a1 - a2 * ro2 + a3 * ro3) * ro3;
    return kc * (a4 - I1);
  }
  if (ro >= 1.0 && ro < 2.0) {
    double ro2 = ro * ro, d = 2.0 - ro, d2 = d * d, d4 = d2 * d2;
    double I2 = -(b1 * ro2 + b2 * d * ro + b3 * d2) * d4;
    return kc * (-I2);
  }
  return 0.0;
}

void cross(const double* u, const double* v, double* w) {   // Vector_Product.f90
  const int iseg[3] = {1, 2, 0};
  for (int i = 0; i < 3; ++i) {
    int j = iseg[i], k = iseg[j];
    w[i] = u[j] * v[k] - u[k] * v[j];
  }
}

int cell_indices(const SimDev& s, int nc, int& i, int& j, int& k) {   // CellIndices.f90
  int ni = s.ncd[0], nj = s.ncd[1];
  int nij = ni * nj;
  k = (nc - 1) / nij + 1;
  int ncij = nc - nij * (k - 1);
  j = (ncij - 1) / ni + 1;
  i = ncij - ni * (j - 1);
  return ncij;
}

// cell_lo, cell_hi (1-based, inclusive; 0 = the whole grid): the x cells of
// a slab of a decomposed simulation, which keeps the whole grid's origin and
// cell size so every particle lies in the cell it has in the whole grid.
int prepare_sim(const SphParams& prm, const SphGeometry& g, int cap, HostSim& hs, int cell_lo = 0,
                int cell_hi = 0) {
  if (prm.dim != 2 && prm.dim != 3) return SPH_ERR_INVALID_ARGUMENT;
  if (!(prm.dx > 0.0) || !(prm.trunc > 0.0) || !(prm.den0 > 0.0) || !(prm.eps > 0.0)) return SPH_ERR_INVALID_ARGUMENT;
  if (!(prm.teta_p >= 0.0) || !(prm.teta_v >= 0.0)) return SPH_ERR_INVALID_ARGUMENT;
  if (prm.precision != SPH_PREC_FP64 && prm.precision != SPH_PREC_FP32C) return SPH_ERR_INVALID_ARGUMENT;
  if (g.n_zones < 0 || (g.n_zones > 0 && !g.zones)) return SPH_ERR_INVALID_ARGUMENT;
  for (int z = 0; z < g.n_zones; ++z) {
    if (g.zones[z].type != SPH_ZONE_FIXE && g.zones[z].type != SPH_ZONE_TAPI) return SPH_ERR_UNSUPPORTED;
    if (g.zones[z].slip_coefficient_mode != 1) return SPH_ERR_UNSUPPORTED;
  }
  hs.prm = prm;
  hs.cap = cap;
  SimDev& s = hs.dev;
  std::memset(&s, 0, sizeof(s));
  s.dim = prm.dim;
  // ReadInput.f90:198-205
  s.h = prm.dx * prm.trunc;
  s.doubleh = 2.0 * s.h;
  s.squareh = s.h * s.h;
  s.square_doubleh = s.doubleh * s.doubleh;
  s.eta = 1.0e-3 * s.h;
  s.eta2 = 1.0e-2 * s.squareh;
  double unosuh = 1.0 / s.h, unosusquareh = 1.0 / s.squareh;
  // Gest_Input.f90:266-289
  double hp = (s.dim == 3) ? (s.h * s.h) * s.h : s.h * s.h;
  s.coefke = ((s.dim == 3) ? 0.477464 : 0.682093) / hp;
  s.coefkacl = ((s.dim == 3) ? 0.074603 : 0.099472) / hp;
  s.ke_coef = s.coefke / s.h;
  s.kacl_coef = s.coefkacl / s.h;
  double r = s.h * 4.0 / prm.dx;
  double rp = (s.dim == 3) ? (r * r) * r : r * r;
  s.nmaxpartj = (int)(prm.coef_nmaxpartj * rp) + 1;
  s.maxcb = (s.dim == 3) ? prm.max_close_bound_faces : kMaxCloseSides;
  if (s.maxcb <= 0) return SPH_ERR_INVALID_ARGUMENT;
  s.dx = prm.dx;
  s.den0 = prm.den0;
  s.eps = prm.eps;
  s.k_over_rho0 = prm.eps / prm.den0;
  s.celerita = std::sqrt(prm.eps / prm.den0);   // ReadInputMedium.f90:156
  s.alfa_mon = prm.alfa_mon;
  s.kin_visc = prm.kin_visc;
  s.p_ref = prm.p_ref;
  for (int d = 0; d < 3; ++d) s.grav[d] = prm.grav[d];
  s.cfl = prm.cfl;
  s.vsc_coeff = prm.vsc_coeff;
  s.pesodt = prm.pesodt;
  if (prm.forcing_period < 0.0 || (prm.forcing_amplitude != 0.0 && !(prm.forcing_period > 0.0)))
    return SPH_ERR_INVALID_ARGUMENT;
  s.forcing_w = prm.forcing_period > 0.0 ? 6.283185307179586 / prm.forcing_period : 0.0;
  s.forcing_aw2 = prm.forcing_amplitude * s.forcing_w * s.forcing_w;
  s.teta_p = prm.teta_p;
  s.teta_v = prm.teta_v;
  // 1st-order consistency: 3D, FP64 form; C1_divu acts only with C1_BE
  // (CalcVarLength.f90:285, Continuity_Equation.f90:201)
  if (prm.c1_be) {
    if (!(prm.invb_det_thresh >= 0.0)) return SPH_ERR_INVALID_ARGUMENT;
    // the 2D matrices are singular (zero y row and column): with a zero
    // threshold the reference's Matrix_Inversion_3x3 divides by det = 0
    if (s.dim == 2 && !(prm.invb_det_thresh > 0.0)) return SPH_ERR_INVALID_ARGUMENT;
  }
  s.c1_be = prm.c1_be ? 1 : 0;
  s.c1_divu = (prm.c1_be && prm.c1_divu) ? 1 : 0;
  s.invb_det_thresh = prm.invb_det_thresh;
  {
    // grad_W_sub.f90:75-88 (3D) with the reference's 14-digit PIGRECO: the
    // per-pair expressions' constant factors, formed as they are there
    const double PIGRECO = 3.14159265358979;
    const double h3 = s.h * s.h * s.h;
    s.c1_w1a = 1.0 / (PIGRECO * h3);
    s.c1_w1b = 3.0 / (4.0 * PIGRECO * h3);
    s.c1_w2 = 15.0 / (64.0 * PIGRECO * h3);
  }
  s.dt_alfa_mon = prm.dt_alfa_mon;
  s.density_thresholds = prm.density_thresholds;
  s.zpmin = 0.05 * s.h;
  // CreaGrid.f90:51-74
  double epsi = 0.01 * prm.dx;
  for (int d = 0; d < 3; ++d) {
    double lo = prm.domain_lo[d] - s.doubleh - epsi;
    double hi = prm.domain_hi[d] + s.doubleh + epsi;
    double dextr = hi - lo;
    s.extr_lo[d] = lo;
    s.ncd[d] = (int)std::lround(dextr / s.doubleh);
    if (s.ncd[d] < 1) return SPH_ERR_INVALID_ARGUMENT;
    s.dcd[d] = dextr / s.ncd[d];
  }
  if (s.dim == 2) s.ncd[1] = 1;
  // IEEE reciprocals of the cell sizes: particle_cell divides by them exactly (div_rn)
  for (int d = 0; d < 3; ++d) s.rcp_dcd[d] = s.dcd[d] > 0.0 ? 1.0 / s.dcd[d] : 0.0;
  // FP32 screening copies (k_rank_permute): the offset f of a particle from
  // the origin o of its cell, in FP32.  A candidate difference is formed as
  // D + (f_i - f_j) with D = (float)(cell index difference * dcd), which is
  // 0 or +-(float)dcd inside the 27-cell block; in z the neighbour-list
  // kernel may instead subtract (A dcdf + f_i) - (B dcdf + f_j), A and B the
  // cell indices less the warp's lowest (|A| <= 6, |B| <= 7), whose rounding
  // is at most (2|A| + 2|B| + 7) 2^-24 dcd <= 33 2^-24 dcd.  Each component
  // is then within eps = 40 * 2^-24 dcd (+ 2^-50 R for the FP64 origins) of
  // x_i - x_j, |x_i - x_j| < 2 dcd, and the FP32 sum of squares adds at most
  // 5 roundings of 2^-24.  Outside twice that band the FP32 value decides
  // the test r^2 <= (2h)^2 exactly as the FP64 one would; inside it the FP64
  // test runs.
  {
    double R2 = 0.0, dmax = 0.0;
    for (int d = 0; d < 3; ++d) {
      if (s.dim == 2 && d == 1) {
        s.dcdf[d] = 0.0f;
        continue;
      }
      double lo = s.extr_lo[d], hi = s.extr_lo[d] + s.dcd[d] * s.ncd[d];
      double rr = std::max(std::fabs(lo), std::fabs(hi));
      R2 += rr * rr;
      dmax = std::max(dmax, s.dcd[d]);
      s.dcdf[d] = (float)s.dcd[d];
    }
    double R = std::sqrt(R2);
    double eps = 40.0 * std::ldexp(dmax, -24) + std::ldexp(R, -50);
    double err = 3.0 * (2.0 * (2.0 * dmax) * eps + eps * eps) + 5.0 * std::ldexp(s.square_doubleh, -24) * 1.01 +
                 1e-14 * s.square_doubleh;
    double band = 2.0 * err;
    s.rr_lo = std::nextafter((float)(s.square_doubleh - band), 0.0f);
    s.rr_hi = std::nextafter((float)(s.square_doubleh + band), 3.0e38f);
    // CreaGrid rounds the cell count to nearest, so a cell can be narrower
    // than 2h; then the list pass masks every hit to the lane's window
    s.narrow_z = s.dcd[2] < s.doubleh ? 1 : 0;
  }
  s.ioff = 0;
  if (cell_lo > 0) {
    if (cell_hi < cell_lo || cell_hi > s.ncd[0]) return SPH_ERR_INVALID_ARGUMENT;
    s.ioff = cell_lo - 1;
    s.ncd[0] = cell_hi - cell_lo + 1;
  }
  long long ncells = (long long)s.ncd[0] * s.ncd[1] * s.ncd[2];
  if (ncells > (1LL << 30)) return SPH_ERR_INVALID_ARGUMENT;
  s.ncells = (int)ncells;
  // ComputeKernelTable.f90:58-71
  s.ktdelta = 2.0 / kKtRows;
  // correctly rounded reciprocals (IEEE division on the host) for the
  // kernels' exact divisions by these constants (div_rn)
  s.rcp_h = 1.0 / s.h;
  s.rcp_squareh = 1.0 / s.squareh;
  s.rcp_ktdelta = 1.0 / s.ktdelta;
  for (int nr = 0; nr <= kKtRows; ++nr) {
    double rob = s.ktdelta * nr;
    s.kerneltab[nr][0] = rob;
    s.kerneltab[nr][1] = iwro2dro(rob);
    s.kerneltab[nr][2] = jdwsrn(rob, 1) * unosusquareh;
    s.kerneltab[nr][3] = jdwsrn(rob, 2) * unosuh;
    s.kerneltab[nr][4] = jdwsrn(rob, 3);
  }
  // ComputeBoundaryIntegralTab.f90:61-86
  hs.bit.assign(kBitRows * 7, 0.0);
  {
    double delta_fi = (kPi / 2.0) / 8;
    double duesendelta_fimz = 2.0 * std::sin(0.5 * delta_fi);
    double delta_teta = (kPi + kPi) / 32;
    double fi = -0.5 * delta_fi;
    int pts = 0;
    for (int i = 1; i <= 8; ++i) {
      fi = fi + delta_fi;
      double teta = -0.5 * delta_teta;
      double zp = -(s.doubleh * std::cos(fi));
      for (int j = 1; j <= 32; ++j) {
        teta = teta + delta_teta;
        double xp = s.doubleh * std::sin(fi) * std::cos(teta);
        double yp = s.doubleh * std::sin(fi) * std::sin(teta);
        double* row = &hs.bit[pts * 7];
        row[0] = xp;
        row[1] = yp;
        row[2] = zp;
        row[3] = delta_teta * duesendelta_fimz * std::sin(fi);
        row[4] = xp / s.doubleh;
        row[5] = yp / s.doubleh;
        row[6] = zp / s.doubleh;
        pts++;
      }
    }
  }
  auto vtx = [&](int id, int d) { return g.vertices[3 * (id - 1) + d]; };
  if (s.dim == 3) {
    // DefineLocalSystemVersors.f90 + DefineBoundaryFaceGeometry3D.f90
    std::vector<FaceGeo> geo(g.n_faces);
    hs.faces.resize(g.n_faces);
    for (int f = 0; f < g.n_faces; ++f) {
      int name[4], nn = 0;
      for (int k = 0; k < 4; ++k) {
        name[k] = g.face_nodes[4 * f + k];
        if (name[k] > 0) {
          if (name[k] > g.n_vertices) return SPH_ERR_INVALID_ARGUMENT;
          nn++;
        }
      }
      if (nn < 3) return SPH_ERR_INVALID_ARGUMENT;
      int zone = g.face_zone[f];
      if (zone < 1 || zone > g.n_zones) return SPH_ERR_INVALID_ARGUMENT;
      FaceGeo& F = geo[f];
      F.nodes = nn;
      F.zone = zone;
      for (int n = 0; n < nn; ++n)
        for (int d = 0; d < 3; ++d) F.GX[n][d] = vtx(name[n], d);
      const int nindex[2][3] = {{1, 2, 3}, {1, 3, 4}};
      int sidek = nn - 2;
      double U1[3], U2[3], RR[3], W12[3], nrm[3], ss[3];
      for (int d = 0; d < 3; ++d) {
        U1[d] = F.GX[nindex[sidek - 1][0] - 1][d] - F.GX[nindex[sidek - 1][2] - 1][d];
        U2[d] = F.GX[nindex[sidek - 1][1] - 1][d] - F.GX[nindex[sidek - 1][2] - 1][d];
      }
      double U1len = std::sqrt(U1[0] * U1[0] + U1[1] * U1[1] + U1[2] * U1[2]);
      for (int d = 0; d < 3; ++d) RR[d] = U1[d] / U1len;
      cross(U1, U2, W12);
      double W12len = std::sqrt(W12[0] * W12[0] + W12[1] * W12[1] + W12[2] * W12[2]);
      if (!(W12len > 1.0e-9)) return SPH_ERR_INVALID_ARGUMENT;
      double area = W12len / (double)(float)(3 - sidek);
      for (int d = 0; d < 3; ++d) nrm[d] = W12[d] / W12len;
      cross(nrm, RR, ss);
      for (int d = 0; d < 3; ++d) {
        F.T[d][0] = RR[d];
        F.T[d][1] = ss[d];
        F.T[d][2] = nrm[d];
      }
      double LX[4][2];
      for (int n = 0; n < nn - 1; ++n)
        for (int i = 0; i < 2; ++i) {
          double a = 0.0;
          for (int j = 0; j < 3; ++j) a = a + F.T[j][i] * (F.GX[n][j] - F.GX[nn - 1][j]);
          LX[n][i] = a;
        }
      LX[nn - 1][0] = 0.0;
      LX[nn - 1][1] = 0.0;
      FaceDev& D = hs.faces[f];
      std::memset(&D, 0, sizeof(D));
      std::memcpy(D.T, F.T, sizeof(D.T));
      for (int d = 0; d < 3; ++d) D.GXref[d] = F.GX[nn - 1][d];
      // LocalNormalCoordinates.f90:59-87 line coefficients
      int fkod = nn - 2;
      const int iseg[3] = {2, 3, 1};
      const int mainod[2][3] = {{1, 2, 3}, {1, 3, 4}};
      D.usu_due_area = 1.0 / ((double)(3 - fkod) * area);
      for (int ii = 1; ii <= 2; ++ii) {
        int jj = iseg[ii - 1], kk = iseg[jj - 1];
        double xj = LX[mainod[fkod - 1][jj - 1] - 1][0], yj = LX[mainod[fkod - 1][jj - 1] - 1][1];
        double xk = LX[mainod[fkod - 1][kk - 1] - 1][0], yk = LX[mainod[fkod - 1][kk - 1] - 1][1];
        D.AA[ii - 1] = xj * yk - xk * yj;
        D.BB[ii - 1] = yj - yk;
        D.CC[ii - 1] = xk - xj;
      }
      D.fkod = fkod;
      const SphZone& z = g.zones[zone - 1];
      for (int d = 0; d < 3; ++d) D.velocity[d] = (z.type == SPH_ZONE_TAPI) ? z.velocity[d] : 0.0;
      D.slip = z.bc_shear_stress_input;
      D.laminar_no_slip_check = z.laminar_no_slip_check;
      D.zone_type = z.type;
    }
    // The boundary quadrature's ring shortcut (face_integrals) needs the
    // computed distances of one ring's points to agree to far better than
    // its 1e-6 margin.  They differ by rounding only, about 2^-49 |L| / h in
    // rob, L the particle's local coordinates: bounded by the grid box's
    // corner farthest from the face's reference vertex.
    double lmax = 0.0;
    for (int f = 0; f < g.n_faces; ++f)
      for (int c = 0; c < 8; ++c) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double corner = s.extr_lo[d] + (((c >> d) & 1) ? s.dcd[d] * s.ncd[d] : 0.0);
          const double u = corner - hs.faces[f].GXref[d];
          d2 += u * u;
        }
        lmax = std::max(lmax, std::sqrt(d2));
      }
    s.ring_skip = (lmax <= 1.0e6 * s.h) ? 1 : 0;
    // CompleteBoundaries3D.f90: BFaceList ordered by zone
    std::vector<int> bface;
    for (int nt = 1; nt <= g.n_zones; ++nt)
      for (int f = 0; f < g.n_faces; ++f)
        if (geo[f].zone == nt) bface.push_back(f + 1);
    // FindBoundaryConvexEdges3D.f90:64-150: for each face of BFaceList, the
    // first later face that shares a side with it, when the shared side is
    // convex (the other face's next node lies behind the first face's
    // plane).  Each face contributes at most one edge, as the reference's
    // loop exits after its first find.  The reference runs the face loop in
    // parallel, so its edge order depends on the threads; this is the order
    // of a serial run.
    hs.edges.clear();
    {
      const int iseg[2][4] = {{2, 3, 1, 0}, {2, 3, 4, 1}};
      auto name = [&](int nf, int i) { return g.face_nodes[4 * (nf - 1) + (i - 1)]; };
      const int nbf = (int)bface.size();
      for (int kf = 0; kf + 1 < nbf; ++kf) {
        const int nf = bface[kf];
        const FaceGeo& F = geo[nf - 1];
        const int nodes = F.nodes, fk = nodes - 2;
        bool found = false;
        for (int kf1 = kf + 1; kf1 < nbf && !found; ++kf1) {
          const int nf1 = bface[kf1];
          const int nodes1 = geo[nf1 - 1].nodes, fk1 = nodes1 - 2;
          for (int i = 1; i <= nodes && !found; ++i) {
            const int nodi = name(nf, i), nodj = name(nf, iseg[fk - 1][i - 1]);
            for (int ii = 1; ii <= nodes1; ++ii) {
              const int jj = iseg[fk1 - 1][ii - 1];
              const int nodii = name(nf1, ii), nodjj = name(nf1, jj);
              if (!((nodi == nodii && nodj == nodjj) || (nodi == nodjj && nodj == nodii))) continue;
              const int nodkk = name(nf1, iseg[fk1 - 1][jj - 1]);
              double zitakk = 0.0;
              for (int sd = 0; sd < 3; ++sd) zitakk = zitakk + F.T[sd][2] * (vtx(nodkk, sd) - F.GX[nodes - 1][sd]);
              if (zitakk < 0.0) {
                EdgeDev E;
                std::memset(&E, 0, sizeof(E));
                E.face[0] = nf;
                E.face[1] = nf1;
                double length2 = 0.0;
                for (int sd = 0; sd < 3; ++sd) {
                  E.gx[sd] = vtx(nodi, sd);
                  const double delta = vtx(nodj, sd) - vtx(nodi, sd);
                  E.comp[sd] = delta;
                  length2 = length2 + delta * delta;
                }
                E.length = std::sqrt(length2);
                hs.edges.push_back(E);
                found = true;
                break;
              }
            }
          }
        }
      }
    }
    s.nedges = (int)hs.edges.size();
    // GridCellBoundaryFacesIntersections3D.f90:89-210, stored by sort key
    hs.cf_count.assign(s.ncells + 1, 0);
    hs.cf_start.assign(s.ncells + 1, 0);
    hs.cf_list.clear();
    std::vector<std::vector<int>> per(s.ncells);
    for (int nc = 1; nc <= s.ncells && !bface.empty(); ++nc) {
      int i, j, k;
      cell_indices(s, nc, i, j, k);
      double cxyz[3][2];
      int idx[3] = {i, j, k};
      for (int d = 0; d < 3; ++d) {
        const int gi = idx[d] + (d == 0 ? s.ioff : 0);   // the whole grid's index
        cxyz[d][0] = s.extr_lo[d] + s.dcd[d] * (gi - 1);
        cxyz[d][1] = s.extr_lo[d] + s.dcd[d] * gi;
      }
      double cn[8][3];
      int nv = 0;
      for (int ii = 0; ii < 2; ++ii)
        for (int jj = 0; jj < 2; ++jj)
          for (int kk = 0; kk < 2; ++kk) {
            cn[nv][0] = cxyz[0][ii];
            cn[nv][1] = cxyz[1][jj];
            cn[nv][2] = cxyz[2][kk];
            nv++;
          }
      std::vector<int>& lst = per[cell_key_local(s, i, j, k)];
      for (int nf : bface) {
        const FaceGeo& F = geo[nf - 1];
        int nodes = F.nodes;
        bool found = true;
        for (int sd = 0; sd < 3 && found; ++sd) {
          int sc[5] = {0, 0, 0, 0, 0};
          for (int no = 0; no < nodes; ++no) {
            double X = F.GX[no][sd];
            if (X < cxyz[sd][0]) sc[0]++;
            else if (X == cxyz[sd][0]) sc[1]++;
            else if (X < cxyz[sd][1]) sc[2]++;
            else if (X == cxyz[sd][1]) sc[3]++;
            else if (X > cxyz[sd][1]) sc[4]++;
          }
          if ((sc[0] + sc[1]) == nodes && !(sc[1] == nodes)) found = false;
          else if ((sc[4] + sc[3]) == nodes && !(sc[3] == nodes)) found = false;
        }
        if (!found) continue;
        int c3[3] = {0, 0, 0};
        for (nv = 0; nv < 8; ++nv) {
          double zita = 0.0;
          for (int sd = 0; sd < 3; ++sd) zita = zita + F.T[sd][2] * (cn[nv][sd] - F.GX[nodes - 1][sd]);
          if (zita < 0.0) c3[0]++;
          else if (zita == 0.0) c3[1]++;
          else c3[2]++;
        }
        if ((c3[0] + c3[1]) == 8 && !(c3[1] == 4)) found = false;
        else if ((c3[2] + c3[1]) == 8 && !(c3[1] == 4)) found = false;
        if (found) {
          if ((int)lst.size() >= prm.max_close_bound_faces) return SPH_ERR_ALLOC;
          lst.push_back(nf);
        }
      }
    }
    for (int key = 0; key < s.ncells; ++key) {
      hs.cf_start[key] = (int)hs.cf_list.size();
      hs.cf_count[key] = (int)per[key].size();
      hs.cf_list.insert(hs.cf_list.end(), per[key].begin(), per[key].end());
    }
    // a cell needs the face search when any of its 27 neighbours is cut
    hs.near.assign(s.ncells + 1, 0);
    for (int k = 1; k <= s.ncd[2]; ++k)
      for (int j = 1; j <= s.ncd[1]; ++j)
        for (int i = 1; i <= s.ncd[0]; ++i) {
          uint8_t any = 0;
          for (int di = -1; di <= 1 && !any; ++di)
            for (int dj = -1; dj <= 1 && !any; ++dj)
              for (int dk = -1; dk <= 1 && !any; ++dk) {
                int a = i + di, bq = j + dj, c = k + dk;
                if (a < 1 || a > s.ncd[0] || bq < 1 || bq > s.ncd[1] || c < 1 || c > s.ncd[2]) continue;
                if (hs.cf_count[cell_key_local(s, a, bq, c)] > 0) any = 1;
              }
          hs.near[cell_key_local(s, i, j, k)] = any;
        }
    s.nfaces = g.n_faces;
  } else {
    // DefineBoundarySideGeometry2D.f90 + BoundaryMassForceMatrix2D.f90 +
    // DefineBoundarySideRelativeAngles2D.f90
    int ns = g.n_sides;
    hs.sides.resize(ns);
    std::vector<double> T11(ns), T31(ns);
    for (int q = 0; q < ns; ++q) {
      int v1 = g.side_vertices[2 * q], v2 = g.side_vertices[2 * q + 1];
      int zone = g.side_zone[q];
      if (v1 < 1 || v2 < 1 || v1 > g.n_vertices || v2 > g.n_vertices || zone < 1 || zone > g.n_zones)
        return SPH_ERR_INVALID_ARGUMENT;
      double Dx = vtx(v2, 0) - vtx(v1, 0);
      double Dz = vtx(v2, 2) - vtx(v1, 2);
      double L = std::sqrt(Dx * Dx + Dz * Dz);
      double sx = Dx / L, sz = Dz / L;
      SideDev& S = hs.sides[q];
      std::memset(&S, 0, sizeof(S));
      S.v1[0] = vtx(v1, 0);
      S.v1[1] = vtx(v1, 2);
      S.sss[0] = sx;
      S.sss[1] = sz;
      S.nnn[0] = -sz;
      S.nnn[1] = sx;
      S.length = L;
      double FiS = 1.0, FiN = 1.0;
      S.RN[0][0] = FiS * sx * sx + FiN * sz * sz;
      S.RN[0][1] = (FiS - FiN) * sx * sz;
      S.RN[1][0] = S.RN[0][1];
      S.RN[1][1] = FiS * sz * sz + FiN * sx * sx;
      const SphZone& z = g.zones[zone - 1];
      for (int d = 0; d < 3; ++d) S.velocity[d] = (z.type == SPH_ZONE_TAPI) ? z.velocity[d] : 0.0;
      S.slip = z.bc_shear_stress_input;
      S.laminar_no_slip_check = z.laminar_no_slip_check;
      S.zone_type = z.type;
      T11[q] = sx;
      T31[q] = sz;
    }
    for (int isi = 0; isi < ns; ++isi) {
      int ksi = 0;
      for (int jsi = 0; jsi < ns; ++jsi)
        if (g.side_vertices[2 * jsi + 1] == g.side_vertices[2 * isi]) { ksi = jsi + 1; break; }
      hs.sides[isi].angle = 0.0;
      if (ksi > 0) {
        double sinangle = T11[ksi - 1] * T31[isi] - T31[ksi - 1] * T11[isi];
        double cosangle = T11[ksi - 1] * T11[isi] + T31[ksi - 1] * T31[isi];
        hs.sides[isi].angle = std::atan2(sinangle, cosangle);
      }
      hs.sides[isi].previous_side = ksi;
    }
    s.nsides = ns;
    hs.cf_count.assign(s.ncells + 1, 0);
    hs.cf_start.assign(s.ncells + 1, 0);
    hs.near.assign(s.ncells + 1, 0);
  }
  return SPH_OK;
}

template <class T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return SPH_ERR_ALLOC;
  }
  return SPH_OK;
}

}  // namespace
}  // namespace sph

using namespace sph;

struct SphHandle {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t stream2 = nullptr;   // the boundary pass beside the lists (step graph)
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t stream3 = nullptr;   // sph_step_download: x, v, m to the host beside the step's end;
                                    // an upload: v, rho, p to the device beside the IC's search
  cudaEvent_t ev_sorted = nullptr;
  cudaEvent_t ev_pos = nullptr, ev_rest = nullptr;   // an upload's two halves
  cudaEvent_t ev_moved = nullptr;   // sph_step_download: the last step's momentum pass done
  int nsims = 0;
  int dim = 3;
  int precision = SPH_PREC_FP64;
  std::vector<HostSim> sims;
  std::vector<int> n_of;            // particles uploaded per simulation
  int total_slots = 0;
  int total_cells = 0;
  int total_faces = 0, total_sides = 0;
  // device memory
  SimDev* d_sims = nullptr;
  SimDyn* d_dyn = nullptr;
  Tile* d_tiles = nullptr;
  FaceDev* d_faces = nullptr;
  SideDev* d_sides = nullptr;
  EdgeDev* d_edges = nullptr;
  double* d_bit = nullptr;
  int *d_cf_start = nullptr, *d_cf_count = nullptr, *d_cf_list = nullptr;
  uint8_t* d_near = nullptr;
  int* d_scan = nullptr;
  int* d_nlist = nullptr;
  int* d_ncount = nullptr;
  int list_cap = 0;
  unsigned long long* d_counters = nullptr;
  double2* d_gq_part = nullptr;     // fluid_global_quantities: per-tile partial sums
  double* d_gq_out = nullptr;       // [nsims][8]
  Particles P{};
  std::vector<void*> owned;
  // caller-order staging
  double *d_cx = nullptr, *d_cv = nullptr, *d_crho = nullptr, *d_cp = nullptr, *d_cm = nullptr;
  double *d_cacc = nullptr, *d_cdden = nullptr;
  int *d_ci1 = nullptr, *d_ci2 = nullptr, *d_ci3 = nullptr;
  double* d_cvals = nullptr;
  size_t cvals_n = 0;
  DevBatch db{};
  cudaGraphExec_t graph = nullptr;
  bool uploaded = false;
  std::vector<SimDyn> h_dyn;
  bool any_teta_v = false;          // some simulation smooths velocities / pressures
  bool any_teta_p = false;
  bool any_c1 = false;              // some simulation renormalises (C1_BE)
  bool any_c1_divu = false;
  size_t device_bytes = 0;          // bytes of the arrays below `owned`
  bool dry = false;                 // size the arrays only (sph_memory_required)
};
// Every entry point that takes a handle runs on the handle's device and
// gives the caller's current device back on return, so a host may hold
// handles on several devices (one per GPU of a node) in one thread.
namespace {
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(const SphHandle* h) {
    if (!h) return;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) { cudaGetLastError(); return; }
    if (cur != h->device && cudaSetDevice(h->device) == cudaSuccess) prev = cur;
    else cudaGetLastError();
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};
}  // namespace


namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return SPH_OK;
  cudaGetLastError();
  return SPH_ERR_CUDA;
}

#define SPH_TRY(x)                  \
  do {                              \
    int _st = (x);                  \
    if (_st != SPH_OK) return _st;  \
  } while (0)
#define SPH_CUDA(x) SPH_TRY(cuda_status(x))

// Handle arrays come from the stream-ordered allocator on the handle's own
// stream, so creating and destroying a handle does not wait for the work
// other handles have queued on the device.
template <class T>
int halloc(SphHandle* h, T** p, size_t n) {
  *p = nullptr;
  size_t bytes = (n == 0 ? 1 : n) * sizeof(T);
  h->device_bytes += bytes;
  if (h->dry) return SPH_OK;
  cudaError_t e = cudaMallocAsync((void**)p, bytes, h->stream);
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return SPH_ERR_ALLOC;
  }
  h->owned.push_back((void*)*p);
  return SPH_OK;
}

// Reads every simulation's device scalars back (CUDA errors only).
int read_dyn(SphHandle* h) {
  SPH_CUDA(cudaMemcpyAsync(h->h_dyn.data(), h->d_dyn, sizeof(SimDyn) * (h->nsims + 1), cudaMemcpyDeviceToHost,
                           h->stream));
  return cuda_status(cudaStreamSynchronize(h->stream));
}

// read_dyn, then the first simulation's fatal status (SPH_OK if none).
int sync_dyn(SphHandle* h) {
  SPH_TRY(read_dyn(h));
  for (int s = 0; s < h->nsims; ++s)
    if (h->h_dyn[s].status != 0) return h->h_dyn[s].status;
  return SPH_OK;
}

void sort_sequence(SphHandle* h, cudaStream_t st) {
  launch_sort_reset(h->db, st);
  launch_bin(h->db, KeyKind::Sort, st);
  launch_removal(h->db, st);
  launch_scan(h->db, h->P.cell_start, st);
  launch_place(h->db, st);
  launch_rank_permute(h->db, st);
}

// CalcVarLength: the neighbour lists and, with C1_BE, the fluid part of
// the renormalisation matrices summed over them.
void lists_pass(SphHandle* h, cudaStream_t st) {
  launch_neighbour_lists(h->db, st);
  if (h->any_c1) launch_renormalisation(h->db, st);
}

void momentum_pass(SphHandle* h, bool fused, cudaStream_t st) {
  if (h->precision == SPH_PREC_FP32C) launch_momentum_f32(h->db, fused, st);
  else launch_momentum(h->db, fused, st);
}

void continuity_pass(SphHandle* h, bool fused, cudaStream_t st) {
  if (h->precision == SPH_PREC_FP32C) launch_continuity_f32(h->db, fused, st);
  else launch_continuity(h->db, fused, st);
}

void refresh_copies(SphHandle* h, cudaStream_t st) {
  if (h->precision == SPH_PREC_FP32C) launch_refresh_f32(h->db, st);
}

// The early half of sph_step_download: positions, velocities and masses
// are final once a step's momentum pass (and velocity smoothing) has run
// (the passes after it write only rho, p and their FP32 copies, and the
// sort only reorders), so their scatter to caller order, from the step's
// record, and their copy to the host run on a third stream beside the sort,
// lists, boundary and continuity passes.  n rows are copied: the count
// before the step, which removals can only lower.  A removal in the step
// renumbers particles: the caller then copies again from the sorted state.
struct EarlyCopy {
  SphState* state;
  int n;
  cudaError_t err;
};

void enqueue_early_copy(SphHandle* h, cudaStream_t st, EarlyCopy& ec) {
  cudaEventRecord(h->ev_moved, st);
  cudaStreamWaitEvent(h->stream3, h->ev_moved, 0);
  cudaStream_t q = h->stream3;
  launch_scratch_to_caller(h->db, h->d_cx, h->d_cv, h->d_cm, q);
  cudaError_t e = cudaGetLastError();
  const size_t o = h->sims[0].dev.p_off, n = (size_t)ec.n;
  SphState* sta = ec.state;
  if (e == cudaSuccess && sta->x) e = cudaMemcpyAsync(sta->x, h->d_cx + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDefault, q);
  if (e == cudaSuccess && sta->v) e = cudaMemcpyAsync(sta->v, h->d_cv + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDefault, q);
  if (e == cudaSuccess && sta->m) e = cudaMemcpyAsync(sta->m, h->d_cm + o, sizeof(double) * n, cudaMemcpyDefault, q);
  ec.err = e;
}

// One whole step.  The boundary data (SA-SPH, FP64, latency-bound) and the
// neighbour lists (FP32 screening, issue-bound) both read the freshly sorted
// state and nothing the other writes, so the boundary pass runs on a second
// stream beside the lists; captured into the step graph this is a fork and
// a join.  The FP64 continuity pass starts its sum from the wall term (the
// reference's order) and waits for both; the FP32c pass sums the pairs
// beside the boundary pass too and adds the wall term after the join.
void step_sequence(SphHandle* h, cudaStream_t st, EarlyCopy* early = nullptr) {
  momentum_pass(h, true, st);
  if (h->any_teta_v) launch_velocity_smoothing(h->db, true, h->precision == SPH_PREC_FP32C, st);
  if (early) enqueue_early_copy(h, st, *early);
  sort_sequence(h, st);
  cudaEventRecord(h->ev_fork, st);
  cudaStreamWaitEvent(h->stream2, h->ev_fork, 0);
  launch_boundary(h->db, h->stream2);
  cudaEventRecord(h->ev_join, h->stream2);
  lists_pass(h, st);
  if (h->precision == SPH_PREC_FP32C) {
    launch_continuity_f32_pairs(h->db, st);
    cudaStreamWaitEvent(st, h->ev_join, 0);
    launch_continuity_f32_finish(h->db, true, st);
  } else {
    cudaStreamWaitEvent(st, h->ev_join, 0);
    continuity_pass(h, true, st);
  }
  if (h->any_teta_p) launch_pressure_smoothing(h->db, h->precision == SPH_PREC_FP32C, st);
  launch_finalize(h->db, 1, st);
}

int build_graph(SphHandle* h) {
  if (h->graph) return SPH_OK;
  cudaGraph_t g = nullptr;
  SPH_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  step_sequence(h, h->stream);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (e != cudaSuccess) return cuda_status(e);
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  return cuda_status(e);
}

// With bytes_out set, nothing touches the device: the arrays are sized,
// their total goes to *bytes_out and no handle is returned.
int create_batch(int nsims, const SphParams* params, const SphGeometry* geoms, const int32_t* caps,
                 SphHandle** out, uint64_t* bytes_out = nullptr, const int32_t* cell_range = nullptr) {
  const bool dry = bytes_out != nullptr;
  if ((!out && !dry) || nsims <= 0 || !params || !geoms || !caps) return SPH_ERR_INVALID_ARGUMENT;
  if (out) *out = nullptr;
  int dev = 0;
  cudaDeviceProp prop{};
  if (!dry) {
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return SPH_ERR_NO_DEVICE; }
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) { cudaGetLastError(); return SPH_ERR_NO_DEVICE; }
    if (prop.major != 10) return SPH_ERR_NO_DEVICE;
  }
  SphHandle* h = new (std::nothrow) SphHandle();
  if (!h) return SPH_ERR_ALLOC;
  h->dry = dry;
  h->device = dev;
  h->nsims = nsims;
  h->dim = params[0].dim;
  h->precision = params[0].precision;
  h->sims.resize(nsims);
  h->n_of.assign(nsims, 0);
  for (int s = 0; s < nsims; ++s) {
    if (params[s].dim != h->dim || params[s].precision != h->precision || caps[s] <= 0) {
      delete h;
      return SPH_ERR_INVALID_ARGUMENT;
    }
    int st = cell_range ? prepare_sim(params[s], geoms[s], caps[s], h->sims[s], cell_range[2 * s], cell_range[2 * s + 1])
                        : prepare_sim(params[s], geoms[s], caps[s], h->sims[s]);
    if (st != SPH_OK) { delete h; return st; }
    if (params[s].teta_v > 1.0e-9) h->any_teta_v = true;
    if (params[s].teta_p > 0.0) h->any_teta_p = true;
    if (h->sims[s].dev.c1_be) h->any_c1 = true;
    if (h->sims[s].dev.c1_divu) h->any_c1_divu = true;
  }
  // layout of the concatenated arrays; simulations start on tile boundaries
  std::vector<Tile> tiles;
  int poff = 0, coff = 0, foff = 0, soff = 0, eoff = 0;
  size_t bdt_cap = 0;
  for (int s = 0; s < nsims; ++s) {
    HostSim& hs = h->sims[s];
    hs.dev.p_off = poff;
    hs.dev.cap = hs.cap;
    hs.dev.cell_off = coff;
    hs.dev.face_off = foff;
    hs.dev.side_off = soff;
    hs.dev.edge_off = eoff;
    // tiles cover the padded segment: every slot, padding included, takes
    // part in the sort, so each simulation's segment stays in place
    for (int t = 0; t < hs.cap; t += kBlock) {
      Tile tl;
      tl.sim = s;
      tl.start = poff + t;
      tl.count = kBlock;
      tl.pad = 0;
      tiles.push_back(tl);
    }
    int padded = (hs.cap + kBlock - 1) / kBlock * kBlock;
    poff += padded;
    coff += hs.dev.ncells + 1;
    foff += (int)hs.faces.size();
    soff += (int)hs.sides.size();
    eoff += (int)hs.edges.size();
    // default: room for three close faces (two close sides) per particle,
    // a box corner's worth; the reference reserves MAXCLOSEBOUNDFACES per
    // particle (Gest_Trans.f90:90), far more than a flow uses
    const size_t quota = hs.prm.bdt_capacity > 0 ? (size_t)hs.prm.bdt_capacity : (size_t)hs.cap * (h->dim == 3 ? 3 : 2);
    if (quota > 0x7fffffff) { delete h; return SPH_ERR_INVALID_ARGUMENT; }
    hs.dev.bdt_quota = (int)quota;
    bdt_cap += quota;
  }
  if (poff >= (1 << 28)) { delete h; return SPH_ERR_INVALID_ARGUMENT; }   // list entries carry 28-bit slots
  h->total_slots = poff;
  h->total_cells = coff;
  h->total_faces = foff;
  h->total_sides = soff;
  int st = SPH_OK;
  cudaError_t e = cudaSuccess;
  if (!dry) {
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) { sph_destroy(h); return cuda_status(e); }
  }
  size_t N = poff, C = coff;
  Particles& P = h->P;
#define A(ptr, n) if (st == SPH_OK) st = halloc(h, &(ptr), (n))
  A(h->d_sims, nsims);
  A(h->d_dyn, nsims + 1);
  A(h->d_tiles, tiles.size());
  A(h->d_faces, foff);
  A(h->d_sides, soff);
  A(h->d_edges, eoff);
  A(h->d_bit, (size_t)nsims * kBitRows * 7);
  A(h->d_cf_start, C);
  A(h->d_cf_count, C);
  A(h->d_near, C);
  A(P.X, N); A(P.XF, N); A(P.VF, N); A(P.RF, N); A(P.RM, N); A(P.V, N); A(P.RP, N); A(P.I, N); A(P.L, N);
  A(P.X2, N); A(P.V2, N); A(P.P2, N); A(P.I2, N); A(P.L2, N);
  A(P.bdt_count, N); A(P.bdt_start, N); A(P.bdt, bdt_cap);
  A(P.key, N); A(P.slot, N); A(P.cell_count, C + 1); A(P.cell_start, C + 1);
  A(P.tmp_src, N); A(P.tmp_id, N); A(P.tmp_key, N);
  A(P.ACC, N); A(P.DDEN, N);
  if (h->precision == SPH_PREC_FP32C) A(P.MSUM, (h->any_c1 ? 12 : 9) * N);   // C1: + the pressure-gradient sums
  if (h->precision == SPH_PREC_FP32C && h->any_teta_v) A(P.VF2, N);
  if (h->any_c1) A(P.BG, 9 * N);
  if (h->any_c1_divu) A(P.BD, 9 * N);
  A(P.out_flag, N); A(P.id_remap, N); A(P.cur_of, N);
  A(h->d_cx, 3 * N); A(h->d_cv, 3 * N); A(h->d_crho, N); A(h->d_cp, N); A(h->d_cm, N);
  A(h->d_cacc, 3 * N); A(h->d_cdden, N);
  A(h->d_ci1, N); A(h->d_ci2, C + 1); A(h->d_ci3, N);
  int nb = (int)((C + 4095) / 4096) + 1;
  A(h->d_scan, nb);
  A(h->d_counters, 4);
  A(h->d_gq_part, tiles.size() * 8);
  A(h->d_gq_out, (size_t)nsims * 8);
  for (int s = 0; s < nsims; ++s) h->list_cap = std::max(h->list_cap, h->sims[s].dev.nmaxpartj);
  h->list_cap = (h->list_cap + 3) / 4 * 4;
  A(h->d_nlist, N * (size_t)h->list_cap);
  A(h->d_ncount, N);
#undef A
  if (st != SPH_OK) { sph_destroy(h); return st; }
  P.bdt_cap = (int)std::min(bdt_cap, (size_t)0x7fffffff);
  P.total_cells = coff;
  P.total_slots = poff;
  // host tables -> device
  std::vector<SimDev> hsd(nsims);
  std::vector<FaceDev> hf;
  std::vector<SideDev> hsi;
  std::vector<EdgeDev> hed;
  std::vector<double> hbit;
  std::vector<int> cfs(C, 0), cfc(C, 0), cfl;
  std::vector<uint8_t> nr(C, 0);
  for (int s = 0; s < nsims; ++s) {
    HostSim& hs = h->sims[s];
    hsd[s] = hs.dev;
    hf.insert(hf.end(), hs.faces.begin(), hs.faces.end());
    hsi.insert(hsi.end(), hs.sides.begin(), hs.sides.end());
    hed.insert(hed.end(), hs.edges.begin(), hs.edges.end());
    hbit.insert(hbit.end(), hs.bit.begin(), hs.bit.end());
    int base = (int)cfl.size();
    for (int k = 0; k < hs.dev.ncells; ++k) {
      cfs[hs.dev.cell_off + k] = base + hs.cf_start[k];
      cfc[hs.dev.cell_off + k] = hs.cf_count[k];
      nr[hs.dev.cell_off + k] = hs.near[k];
    }
    cfl.insert(cfl.end(), hs.cf_list.begin(), hs.cf_list.end());
  }
  if (st == SPH_OK) st = halloc(h, &h->d_cf_list, cfl.size());
  if (dry) {
    *bytes_out = h->device_bytes;
    delete h;
    return SPH_OK;
  }
  if (st != SPH_OK) { sph_destroy(h); return st; }
  cudaStream_t q = h->stream;
  std::vector<SimDyn> dyn0(nsims + 1);
  std::memset(dyn0.data(), 0, sizeof(SimDyn) * (nsims + 1));
  for (auto& d : dyn0) d.dtmin_bits = 0x7FF0000000000000ull;
  h->h_dyn = dyn0;
  double bit2d[22][6];
  for (int i = 0; i < 22; ++i)
    for (int j = 0; j < 6; ++j) bit2d[i][j] = (double)kBit2dLiterals[i][j];
  e = cudaMemcpyAsync(h->d_sims, hsd.data(), sizeof(SimDev) * nsims, cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_dyn, dyn0.data(), sizeof(SimDyn) * (nsims + 1), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess && !hf.empty()) e = cudaMemcpyAsync(h->d_faces, hf.data(), sizeof(FaceDev) * hf.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess && !hsi.empty()) e = cudaMemcpyAsync(h->d_sides, hsi.data(), sizeof(SideDev) * hsi.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess && !hed.empty()) e = cudaMemcpyAsync(h->d_edges, hed.data(), sizeof(EdgeDev) * hed.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_bit, hbit.data(), sizeof(double) * hbit.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_cf_start, cfs.data(), sizeof(int) * C, cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_cf_count, cfc.data(), sizeof(int) * C, cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h->d_near, nr.data(), C, cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess && !cfl.empty()) e = cudaMemcpyAsync(h->d_cf_list, cfl.data(), sizeof(int) * cfl.size(), cudaMemcpyHostToDevice, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.cell_count, 0, sizeof(int) * (C + 1), q);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.out_flag, 0, N, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.bdt_count, 0, sizeof(int) * N, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.ACC, 0, sizeof(double4) * N, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(P.DDEN, 0, sizeof(double) * N, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_counters, 0, sizeof(unsigned long long) * 4, q);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_ncount, 0, sizeof(int) * N, q);
  if (e == cudaSuccess) upload_bit2d(&bit2d[0][0], q);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  if (e != cudaSuccess) { sph_destroy(h); return cuda_status(e); }
  DevBatch& b = h->db;
  b.sims = h->d_sims;
  b.dyn = h->d_dyn;
  b.tiles = h->d_tiles;
  b.ntiles = (int)tiles.size();
  b.nsims = nsims;
  b.dim = h->dim;
  b.P = P;
  b.faces = h->d_faces;
  b.sides = h->d_sides;
  b.edges = h->d_edges;
  b.bit = h->d_bit;
  b.cf_start = h->d_cf_start;
  b.cf_count = h->d_cf_count;
  b.cf_list = h->d_cf_list;
  b.cell_near = h->d_near;
  b.scan_block_sums = h->d_scan;
  b.counters = h->d_counters;
  b.nlist = h->d_nlist;
  b.ncount = h->d_ncount;
  b.list_cap4 = h->list_cap / 4;
  b.scan_nblocks = nb;
  b.grid_blocks = prop.multiProcessorCount * 8;
  b.sms = prop.multiProcessorCount;
  for (int c = 0; c < kGridClasses; ++c) b.grid[c] = 0;
  b.c1 = h->any_c1 ? 1 : 0;
  b.c1_divu = h->any_c1_divu ? 1 : 0;
  b.mom_batch = 0;
  b.con_batch = 0;
  *out = h;
  return SPH_OK;
}

// The caller's arrays may be host memory (pageable or page-locked) or
// device memory of the handle's device: the copies take the direction from
// the pointers (unified addressing), so a host that keeps its state on the
// device (e.g. a slab exchange done with device tensors) never stages it
// through the host.
// The positions and masses of simulation `sim` (what the sort needs), on
// the handle's stream.
int upload_positions(SphHandle* h, int sim, const SphState* st) {
  if (!h || !st || sim < 0 || sim >= h->nsims) return SPH_ERR_INVALID_ARGUMENT;
  HostSim& hs = h->sims[sim];
  if (st->n < 0 || st->n > hs.cap || !st->x || !st->v || !st->rho || !st->p || !st->m) return SPH_ERR_INVALID_ARGUMENT;
  size_t o = hs.dev.p_off, n = st->n;
  cudaStream_t q = h->stream;
  SPH_CUDA(cudaMemcpyAsync(h->d_cx + 3 * o, st->x, sizeof(double) * 3 * n, cudaMemcpyDefault, q));
  SPH_CUDA(cudaMemcpyAsync(h->d_cm + o, st->m, sizeof(double) * n, cudaMemcpyDefault, q));
  h->n_of[sim] = st->n;
  return SPH_OK;
}

// Its velocities, densities and pressures, on stream q (after
// upload_positions has checked the state).
int upload_rest(SphHandle* h, int sim, const SphState* st, cudaStream_t q) {
  size_t o = h->sims[sim].dev.p_off, n = st->n;
  SPH_CUDA(cudaMemcpyAsync(h->d_cv + 3 * o, st->v, sizeof(double) * 3 * n, cudaMemcpyDefault, q));
  SPH_CUDA(cudaMemcpyAsync(h->d_crho + o, st->rho, sizeof(double) * n, cudaMemcpyDefault, q));
  SPH_CUDA(cudaMemcpyAsync(h->d_cp + o, st->p, sizeof(double) * n, cudaMemcpyDefault, q));
  return SPH_OK;
}

int upload_sim(SphHandle* h, int sim, const SphState* st) {
  SPH_TRY(upload_positions(h, sim, st));
  return upload_rest(h, sim, st, h->stream);
}

// The third stream and its events, made on first use.
int ensure_stream3(SphHandle* h) {
  if (h->stream3) return SPH_OK;
  SPH_CUDA(cudaStreamCreateWithFlags(&h->stream3, cudaStreamNonBlocking));
  SPH_CUDA(cudaEventCreateWithFlags(&h->ev_sorted, cudaEventDisableTiming));
  SPH_CUDA(cudaEventCreateWithFlags(&h->ev_pos, cudaEventDisableTiming));
  SPH_CUDA(cudaEventCreateWithFlags(&h->ev_rest, cudaEventDisableTiming));
  SPH_CUDA(cudaEventCreateWithFlags(&h->ev_moved, cudaEventDisableTiming));
  return SPH_OK;
}

// Upload and IC of all simulations: sort, lists, boundary data, IC time
// step.  The positions and masses go first, and the sort, the lists and the
// boundary data run on them while the velocities, densities and pressures
// are still being copied (stream 3); those are gathered into the sorted
// order once both the copy and the sort are done, before the renormalisation
// matrices and the time step that read them.  The boundary pass runs beside
// the lists, as in the step.  The same results as one stream in sequence.
int upload_and_initialise(SphHandle* h, const SphState* states) {
  SPH_TRY(ensure_stream3(h));
  cudaStream_t q = h->stream, q3 = h->stream3;
  for (int s = 0; s < h->nsims; ++s) SPH_TRY(upload_positions(h, s, &states[s]));
  for (int s = 0; s < h->nsims; ++s) {
    std::memset(&h->h_dyn[s], 0, sizeof(SimDyn));
    h->h_dyn[s].nag = h->n_of[s];
    h->h_dyn[s].dtmin_bits = 0x7FF0000000000000ull;
    h->h_dyn[s].t_end = 0.0;
  }
  std::memset(&h->h_dyn[h->nsims], 0, sizeof(SimDyn));
  SPH_CUDA(cudaMemcpyAsync(h->d_dyn, h->h_dyn.data(), sizeof(SimDyn) * (h->nsims + 1), cudaMemcpyHostToDevice, q));
  launch_init_positions(h->db, h->d_cx, h->d_cm, q);
  SPH_CUDA(cudaEventRecord(h->ev_pos, q));
  SPH_CUDA(cudaStreamWaitEvent(q3, h->ev_pos, 0));
  for (int s = 0; s < h->nsims; ++s) SPH_TRY(upload_rest(h, s, &states[s], q3));
  launch_init_rest(h->db, h->d_cv, h->d_crho, h->d_cp, q3);
  launch_sort_reset(h->db, q);
  launch_bin(h->db, KeyKind::Sort, q);
  launch_removal(h->db, q);
  launch_scan(h->db, h->P.cell_start, q);
  launch_place(h->db, q);
  launch_rank_permute_positions(h->db, q);
  SPH_CUDA(cudaEventRecord(h->ev_sorted, q));
  SPH_CUDA(cudaStreamWaitEvent(q3, h->ev_sorted, 0));
  launch_rank_permute_rest(h->db, q3);
  SPH_CUDA(cudaEventRecord(h->ev_rest, q3));
  SPH_CUDA(cudaEventRecord(h->ev_fork, q));
  SPH_CUDA(cudaStreamWaitEvent(h->stream2, h->ev_fork, 0));
  launch_boundary(h->db, h->stream2);
  SPH_CUDA(cudaEventRecord(h->ev_join, h->stream2));
  launch_neighbour_lists(h->db, q);
  SPH_CUDA(cudaStreamWaitEvent(q, h->ev_join, 0));
  SPH_CUDA(cudaStreamWaitEvent(q, h->ev_rest, 0));
  if (h->any_c1) launch_renormalisation(h->db, q);
  launch_dt_reduce(h->db, q);
  launch_finalize(h->db, 0, q);
  SPH_CUDA(cudaGetLastError());
  h->uploaded = true;
  return sync_dyn(h);
}

}  // namespace

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

int sph_create(const SphParams* params, const SphGeometry* geometry, int32_t n_capacity, SphHandle** out) {
  if (!params || !geometry) return SPH_ERR_INVALID_ARGUMENT;
  return create_batch(1, params, geometry, &n_capacity, out);
}

int sph_batch_create(int32_t nsims, const SphParams* params, const SphGeometry* geometries,
                     const int32_t* n_capacity, SphHandle** out) {
  return create_batch(nsims, params, geometries, n_capacity, out);
}

void sph_destroy(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (void* p : h->owned) cudaFreeAsync(p, h->stream);
  if (h->stream) {
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
  }
  if (h->stream2) cudaStreamDestroy(h->stream2);
  if (h->stream3) {
    cudaStreamSynchronize(h->stream3);
    cudaStreamDestroy(h->stream3);
  }
  if (h->ev_sorted) cudaEventDestroy(h->ev_sorted);
  if (h->ev_pos) cudaEventDestroy(h->ev_pos);
  if (h->ev_rest) cudaEventDestroy(h->ev_rest);
  if (h->ev_moved) cudaEventDestroy(h->ev_moved);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  cudaGetLastError();
  delete h;
}

int sph_memory_required(int32_t nsims, const SphParams* params, const SphGeometry* geometries,
                        const int32_t* n_capacity, uint64_t* bytes) {
  if (!bytes) return SPH_ERR_INVALID_ARGUMENT;
  *bytes = 0;
  return create_batch(nsims, params, geometries, n_capacity, nullptr, bytes);
}

int sph_idle(SphHandle* h, int32_t* idle) {
  DeviceGuard dev_guard_(h);
  if (!h || !idle) return SPH_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamQuery(h->stream);
  if (e == cudaErrorNotReady) {
    *idle = 0;
    return SPH_OK;
  }
  *idle = 1;
  return cuda_status(e);
}

int sph_upload(SphHandle* h, const SphState* state) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_upload: IC (OrdGrid1, CalcVarLength, ComputeBoundaryDataTab, time_step_duration)");
  if (!h || h->nsims != 1 || !state) return SPH_ERR_INVALID_ARGUMENT;
  return upload_and_initialise(h, state);
}

int sph_batch_upload(SphHandle* h, int32_t nsims, const SphState* states) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_batch_upload: IC of every simulation");
  if (!h || nsims != h->nsims || !states) return SPH_ERR_INVALID_ARGUMENT;
  return upload_and_initialise(h, states);
}

int sph_batch_set_end_time(SphHandle* h, int32_t sim, double t_end) {
  DeviceGuard dev_guard_(h);
  if (!h || sim < 0 || sim >= h->nsims || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  SPH_CUDA(cudaMemcpyAsync(&h->d_dyn[sim].t_end, &t_end, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return cuda_status(cudaStreamSynchronize(h->stream));
}

// Copies one simulation's state back.  Its result is that simulation's own
// status (another member's failure does not stop the download of a healthy
// one); a failed or cancelled member's state is still copied, for
// inspection, and its code returned.
static int download_impl(SphHandle* h, int sim, SphState* state, double* acc, double* dden) {
  if (!h || !h->uploaded || sim < 0 || sim >= h->nsims) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(read_dyn(h));
  HostSim& hs = h->sims[sim];
  int n = h->h_dyn[sim].nag;
  cudaStream_t q = h->stream;
  launch_to_caller(h->db, h->d_cx, h->d_cv, h->d_crho, h->d_cp, h->d_cm, acc ? h->d_cacc : nullptr,
                   dden ? h->d_cdden : nullptr, q);
  SPH_CUDA(cudaGetLastError());
  size_t o = hs.dev.p_off;
  if (state) {
    state->n = n;
    if (state->x) SPH_CUDA(cudaMemcpyAsync(state->x, h->d_cx + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDefault, q));
    if (state->v) SPH_CUDA(cudaMemcpyAsync(state->v, h->d_cv + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDefault, q));
    if (state->rho) SPH_CUDA(cudaMemcpyAsync(state->rho, h->d_crho + o, sizeof(double) * n, cudaMemcpyDefault, q));
    if (state->p) SPH_CUDA(cudaMemcpyAsync(state->p, h->d_cp + o, sizeof(double) * n, cudaMemcpyDefault, q));
    if (state->m) SPH_CUDA(cudaMemcpyAsync(state->m, h->d_cm + o, sizeof(double) * n, cudaMemcpyDefault, q));
  }
  if (acc) SPH_CUDA(cudaMemcpyAsync(acc, h->d_cacc + 3 * o, sizeof(double) * 3 * n, cudaMemcpyDefault, q));
  if (dden) SPH_CUDA(cudaMemcpyAsync(dden, h->d_cdden + o, sizeof(double) * n, cudaMemcpyDefault, q));
  SPH_CUDA(cudaStreamSynchronize(q));
  return h->h_dyn[sim].status;
}

int sph_download(SphHandle* h, SphState* state) {
  DeviceGuard dev_guard_(h);
  if (!h || h->nsims != 1 || !state) return SPH_ERR_INVALID_ARGUMENT;
  return download_impl(h, 0, state, nullptr, nullptr);
}

int sph_batch_download(SphHandle* h, int32_t sim, SphState* state) {
  DeviceGuard dev_guard_(h);
  return download_impl(h, sim, state, nullptr, nullptr);
}

static void fill_info(SphHandle* h, int sim, SphStepInfo* info) {
  const SimDyn& d = h->h_dyn[sim];
  info->time = d.time;
  info->dt = d.dt_prev;
  info->step = d.step;
  info->n = d.nag;
  info->warnings = d.warnings;
  info->max_neighbours = d.max_neigh;
}

int sph_step(SphHandle* h, int32_t nsteps, SphStepInfo* info) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_step: time_step_loop");
  if (!h || !h->uploaded || nsteps < 0) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(build_graph(h));
  for (int s = 0; s < nsteps; ++s) SPH_CUDA(cudaGraphLaunch(h->graph, h->stream));
  SPH_TRY(sync_dyn(h));
  if (info) fill_info(h, 0, info);
  return SPH_OK;
}

// nsteps steps, then the state in caller order, as sph_step followed by
// sph_download, with the last step's positions, velocities and masses
// copied to the host while that step's sort, lists, boundary data and
// continuity pass still run (see enqueue_early_copy).  The last step is launched
// without the graph so that the copy can start inside it.
int sph_step_download(SphHandle* h, int32_t nsteps, SphState* state) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_step_download: time_step_loop + pg(:) to the host");
  if (!h || !h->uploaded || h->nsims != 1 || nsteps < 0 || !state) return SPH_ERR_INVALID_ARGUMENT;
  if (nsteps == 0) return download_impl(h, 0, state, nullptr, nullptr);
  SPH_TRY(build_graph(h));
  SPH_TRY(ensure_stream3(h));
  for (int s = 0; s + 1 < nsteps; ++s) SPH_CUDA(cudaGraphLaunch(h->graph, h->stream));
  // rows to copy early: the count the host last read back, which the steps
  // enqueued since can only have lowered (removals), so no wait is needed
  // between the graph launches and the last step's launches
  EarlyCopy ec{state, h->h_dyn[0].nag, cudaSuccess};
  cudaStream_t q = h->stream;
  step_sequence(h, q, &ec);
  launch_to_caller(h->db, nullptr, nullptr, h->d_crho, h->d_cp, nullptr, nullptr, nullptr, q);
  cudaError_t e = cudaGetLastError();
  const size_t o = h->sims[0].dev.p_off, n = (size_t)ec.n;
  if (e == cudaSuccess && state->rho) e = cudaMemcpyAsync(state->rho, h->d_crho + o, sizeof(double) * n, cudaMemcpyDefault, q);
  if (e == cudaSuccess && state->p) e = cudaMemcpyAsync(state->p, h->d_cp + o, sizeof(double) * n, cudaMemcpyDefault, q);
  cudaError_t e3 = cudaStreamSynchronize(h->stream3);
  if (e == cudaSuccess) e = ec.err;
  if (e == cudaSuccess) e = e3;
  SPH_TRY(sync_dyn(h));
  if (e != cudaSuccess) return cuda_status(e);
  state->n = h->h_dyn[0].nag;
  if (state->n != ec.n && (state->x || state->v || state->m)) {
    // particles were removed (and renumbered): the rows again, from the
    // sorted state in the final numbering
    launch_to_caller(h->db, h->d_cx, h->d_cv, nullptr, nullptr, h->d_cm, nullptr, nullptr, q);
    SPH_CUDA(cudaGetLastError());
    const size_t m = (size_t)state->n;
    if (state->x) SPH_CUDA(cudaMemcpyAsync(state->x, h->d_cx + 3 * o, sizeof(double) * 3 * m, cudaMemcpyDefault, q));
    if (state->v) SPH_CUDA(cudaMemcpyAsync(state->v, h->d_cv + 3 * o, sizeof(double) * 3 * m, cudaMemcpyDefault, q));
    if (state->m) SPH_CUDA(cudaMemcpyAsync(state->m, h->d_cm + o, sizeof(double) * m, cudaMemcpyDefault, q));
    SPH_CUDA(cudaStreamSynchronize(q));
  }
  return SPH_OK;
}

// Enqueue steps without waiting (the caller synchronises through sph_sync).
int sph_step_async(SphHandle* h, int32_t nsteps) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_step_async: time_step_loop (enqueued)");
  if (!h || !h->uploaded || nsteps < 0) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(build_graph(h));
  for (int s = 0; s < nsteps; ++s) SPH_CUDA(cudaGraphLaunch(h->graph, h->stream));
  return SPH_OK;
}

int sph_sync(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  if (!h) return SPH_ERR_INVALID_ARGUMENT;
  return sync_dyn(h);
}

int sph_batch_info(SphHandle* h, int32_t sim, SphStepInfo* info, int32_t* frozen) {
  DeviceGuard dev_guard_(h);
  if (!h || sim < 0 || sim >= h->nsims || !info) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  fill_info(h, sim, info);
  if (frozen) *frozen = h->h_dyn[sim].frozen;
  return SPH_OK;
}

void* sph_stream(SphHandle* h) { return h ? (void*)h->stream : nullptr; }

// All simulations' progress in one read-back: frozen flag, time, steps and
// fatal status.  A member's failure is reported in status[], not as the
// call's result, so a server can retire it and keep the others running.
int sph_batch_status(SphHandle* h, int32_t* frozen, double* time, int32_t* steps, int32_t* status) {
  DeviceGuard dev_guard_(h);
  if (!h) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(read_dyn(h));
  for (int s = 0; s < h->nsims; ++s) {
    if (frozen) frozen[s] = h->h_dyn[s].frozen;
    if (time) time[s] = h->h_dyn[s].time;
    if (steps) steps[s] = h->h_dyn[s].step;
    if (status) status[s] = h->h_dyn[s].status;
  }
  return SPH_OK;
}

// The device the next sph_create / sph_batch_create / sph_create_slab of
// this host thread builds its handle on (cudaSetDevice); every call on a
// handle then runs on the handle's own device whatever the current one.
int sph_select_device(int32_t device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return SPH_ERR_NO_DEVICE; }
  if (device < 0 || device >= n) return SPH_ERR_INVALID_ARGUMENT;
  return cuda_status(cudaSetDevice(device));
}

// ------------------------------------------------------------------- slabs
int sph_create_slab(const SphParams* params, const SphGeometry* geometry, int32_t n_capacity, int32_t cell_lo,
                    int32_t cell_hi, SphHandle** out) {
  if (!params || !geometry || cell_lo < 1) return SPH_ERR_INVALID_ARGUMENT;
  // the renormalisation matrices and the smoothing passes need exchanges
  // this decomposition does not make; the time-step override assumes pesodt 0
  if (params->c1_be || params->teta_v > 1.0e-9 || params->teta_p > 0.0 || params->pesodt != 0.0)
    return SPH_ERR_UNSUPPORTED;
  const int32_t range[2] = {cell_lo, cell_hi};
  return create_batch(1, params, geometry, &n_capacity, out, nullptr, range);
}

// A new particle set with the simulation's clock kept: OrdGrid1, the
// neighbour lists and ComputeBoundaryDataTab on it (the search of
// time_step_loop.f90:286-324), no time-step evaluation.
int sph_replace_particles(SphHandle* h, const SphState* state, const int32_t* laminar) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_replace_particles: OrdGrid1, CalcVarLength, ComputeBoundaryDataTab");
  if (!h || !h->uploaded || h->nsims != 1 || !state) return SPH_ERR_INVALID_ARGUMENT;
  if (h->any_c1) return SPH_ERR_UNSUPPORTED;
  SPH_TRY(read_dyn(h));
  SPH_TRY(upload_sim(h, 0, state));
  h->h_dyn[0].nag = state->n;
  cudaStream_t q = h->stream;
  SPH_CUDA(cudaMemcpyAsync(h->d_dyn, h->h_dyn.data(), sizeof(SimDyn), cudaMemcpyHostToDevice, q));
  if (laminar && state->n > 0)
    SPH_CUDA(cudaMemcpyAsync(h->d_ci1, laminar, sizeof(int32_t) * state->n, cudaMemcpyDefault, q));
  launch_init_from_caller(h->db, h->d_cx, h->d_cv, h->d_crho, h->d_cp, h->d_cm, q);
  sort_sequence(h, q);
  if (laminar && state->n > 0) launch_load_laminar(h->db, h->d_ci1, q);
  launch_boundary(h->db, q);
  lists_pass(h, q);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_set_time_step(SphHandle* h, double dt) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || !(dt > 0.0)) return SPH_ERR_INVALID_ARGUMENT;
  for (int s = 0; s < h->nsims; ++s)
    if (h->sims[s].prm.pesodt != 0.0) return SPH_ERR_UNSUPPORTED;
  launch_set_dt(h->db, dt, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

// ------------------------------------------------------------- checkpoint
int sph_get_clock(SphHandle* h, SphClock* clock) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || !clock) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  const SimDyn& d = h->h_dyn[0];
  clock->time = d.time;
  clock->dt = d.dt;
  clock->dt_prev = d.dt_prev;
  clock->dt_average = d.dt_average;
  clock->step = d.step;
  clock->reserved = 0;
  return SPH_OK;
}

int sph_set_clock(SphHandle* h, const SphClock* clock, const int32_t* laminar) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || !clock) return SPH_ERR_INVALID_ARGUMENT;
  if (h->any_c1) return SPH_ERR_UNSUPPORTED;
  if (!(clock->dt > 0.0) || !(clock->dt_prev > 0.0) || clock->step < 0 || !(clock->time >= 0.0))
    return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  const int n = h->h_dyn[0].nag;
  cudaStream_t q = h->stream;
  if (laminar && n > 0)
    SPH_CUDA(cudaMemcpyAsync(h->d_ci1, laminar, sizeof(int32_t) * n, cudaMemcpyDefault, q));
  launch_set_clock(h->db, clock->time, clock->step, clock->dt, clock->dt_prev, clock->dt_average,
                   laminar && n > 0 ? h->d_ci1 : nullptr, q);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

// Stops simulation `sim` from the next enqueued launch on (stream-ordered,
// no wait): it freezes with status SPH_CANCELLED and keeps its state.
int sph_batch_cancel(SphHandle* h, int32_t sim) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || sim < 0 || sim >= h->nsims) return SPH_ERR_INVALID_ARGUMENT;
  launch_cancel(h->db, sim, h->stream);
  return cuda_status(cudaGetLastError());
}

int sph_get_diagnostics(SphHandle* h, SphDiagnostics* diag) {
  DeviceGuard dev_guard_(h);
  if (!h || !diag) return SPH_ERR_INVALID_ARGUMENT;
  int st = sync_dyn(h);
  const SimDyn& d = h->h_dyn[0];
  const SimDev& s = h->sims[0].dev;
  diag->warnings = d.warnings;
  diag->status = d.status;
  diag->removed_out_of_grid = d.removed_total;
  diag->ncbf_max = d.ncbf_max;
  diag->bdt_entries = h->h_dyn[h->nsims].bdt_used;
  diag->nmaxpartj = s.nmaxpartj;
  for (int k = 0; k < 3; ++k) diag->grid_ncd[k] = s.ncd[k];
  diag->n_cells = s.ncells;
  return st == SPH_ERR_CUDA ? st : SPH_OK;
}

// ---------------------------------------------------------------- fine-grained
int sph_time_step_duration(SphHandle* h, double* dt_out) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("time_step_duration");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  if (dt_out) *dt_out = h->h_dyn[0].dt;
  return SPH_OK;
}

int sph_rhs_momentum(SphHandle* h, double* acc_out) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("RHS_momentum_equation");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  momentum_pass(h, false, h->stream);
  SPH_CUDA(cudaGetLastError());
  if (acc_out) return download_impl(h, 0, nullptr, acc_out, nullptr);
  return sync_dyn(h);
}

int sph_leapfrog_momentum(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("Leapfrog_momentum");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_leapfrog_momentum(h->db, h->stream);
  if (h->any_teta_v) launch_velocity_smoothing(h->db, false, h->precision == SPH_PREC_FP32C, h->stream);
  refresh_copies(h, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_leapfrog_trajectories(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("Leapfrog_trajectories");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_leapfrog_trajectories(h->db, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_ord_grid(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("OrdGrid1 + CalcVarLength");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_stage(h->db, h->stream);
  sort_sequence(h, h->stream);
  lists_pass(h, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_boundary_data_tab(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("ComputeBoundaryDataTab");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_boundary(h->db, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_continuity(SphHandle* h, double* dden_out) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("SASPH_continuity + Continuity_Equation");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  continuity_pass(h, false, h->stream);
  SPH_CUDA(cudaGetLastError());
  if (dden_out) return download_impl(h, 0, nullptr, nullptr, dden_out);
  return sync_dyn(h);
}

int sph_leapfrog_continuity(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("Leapfrog_continuity");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_leapfrog_continuity(h->db, h->stream);
  refresh_copies(h, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

int sph_eos(SphHandle* h) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("EoS_fluid_loop + time_step_duration");
  if (!h || !h->uploaded) return SPH_ERR_INVALID_ARGUMENT;
  launch_eos(h->db, h->stream);
  if (h->any_teta_p) launch_pressure_smoothing(h->db, h->precision == SPH_PREC_FP32C, h->stream);
  refresh_copies(h, h->stream);
  launch_dt_reduce(h->db, h->stream);
  launch_finalize(h->db, 1, h->stream);
  SPH_CUDA(cudaGetLastError());
  return sync_dyn(h);
}

// ------------------------------------------------------- global quantities
// fluid_global_quantities.f90:59-72 for simulation `sim` (out[8]) or, with
// sim = -1, for every simulation of the handle (out[nsims][8]).
int sph_global_quantities(SphHandle* h, int32_t sim, double* out) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("fluid_global_quantities");
  if (!h || !h->uploaded || !out || sim < -1 || sim >= h->nsims) return SPH_ERR_INVALID_ARGUMENT;
  cudaStream_t q = h->stream;
  launch_global_quantities(h->db, h->d_gq_part, h->d_gq_out, q);
  SPH_CUDA(cudaGetLastError());
  const size_t first = sim < 0 ? 0 : (size_t)sim, count = sim < 0 ? (size_t)h->nsims : 1;
  SPH_CUDA(cudaMemcpyAsync(out, h->d_gq_out + 8 * first, sizeof(double) * 8 * count, cudaMemcpyDeviceToHost, q));
  return sync_dyn(h);
}

// ---------------------------------------------------------------- verification
int sph_dump_grid(SphHandle* h, int32_t* cella, int32_t* icont, int32_t* npartord) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  int n = h->h_dyn[0].nag;
  int ncells = h->sims[0].dev.ncells;
  cudaStream_t q = h->stream;
  if (cella) {
    launch_dump_cella(h->db, h->d_ci1, q);
    SPH_CUDA(cudaMemcpyAsync(cella, h->d_ci1, sizeof(int) * n, cudaMemcpyDeviceToHost, q));
  }
  if (icont || npartord) {
    launch_sort_reset(h->db, q);
    launch_bin(h->db, KeyKind::Reference, q);
    launch_scan(h->db, h->d_ci2, q);
    launch_rank_reference(h->db, h->d_ci2, h->d_ci3, q);
    SPH_CUDA(cudaGetLastError());
    if (icont) {
      std::vector<int> cs(ncells + 1);
      SPH_CUDA(cudaMemcpyAsync(cs.data(), h->d_ci2, sizeof(int) * (ncells + 1), cudaMemcpyDeviceToHost, q));
      SPH_CUDA(cudaStreamSynchronize(q));
      for (int c = 0; c <= ncells; ++c) icont[c] = cs[c] + 1;   // Icont is 1-based
    }
    if (npartord) SPH_CUDA(cudaMemcpyAsync(npartord, h->d_ci3, sizeof(int) * n, cudaMemcpyDeviceToHost, q));
  }
  return cuda_status(cudaStreamSynchronize(q));
}

int sph_dump_neighbours(SphHandle* h, int32_t nmaxj, int32_t* counts, int32_t* lists) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || nmaxj <= 0 || !counts || !lists) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  int n = h->h_dyn[0].nag;
  int* dl = nullptr;
  SPH_TRY(dalloc(&dl, (size_t)n * nmaxj));
  cudaStream_t q = h->stream;
  cudaMemsetAsync(dl, 0, sizeof(int) * (size_t)n * nmaxj, q);
  launch_dump_neighbours(h->db, nmaxj, h->d_ci1, dl, q);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(counts, h->d_ci1, sizeof(int) * n, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(lists, dl, sizeof(int) * (size_t)n * nmaxj, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  cudaFree(dl);
  return cuda_status(e);
}

int sph_dump_boundary(SphHandle* h, int32_t max_per, int32_t* ncb, int32_t* clobonum, double* values) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || max_per <= 0 || !ncb || !clobonum || !values) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  int n = h->h_dyn[0].nag;
  int *dc = nullptr;
  double* dv = nullptr;
  SPH_TRY(dalloc(&dc, (size_t)n * max_per));
  if (dalloc(&dv, (size_t)n * max_per * 20) != SPH_OK) { cudaFree(dc); return SPH_ERR_ALLOC; }
  cudaStream_t q = h->stream;
  cudaMemsetAsync(dc, 0, sizeof(int) * (size_t)n * max_per, q);
  cudaMemsetAsync(dv, 0, sizeof(double) * (size_t)n * max_per * 20, q);
  launch_dump_boundary(h->db, max_per, h->d_ci1, dc, dv, q);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(ncb, h->d_ci1, sizeof(int) * n, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(clobonum, dc, sizeof(int) * (size_t)n * max_per, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaMemcpyAsync(values, dv, sizeof(double) * (size_t)n * max_per * 20, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  cudaFree(dc);
  cudaFree(dv);
  return cuda_status(e);
}

int sph_dump_laminar(SphHandle* h, int32_t* flags) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || !flags) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  int n = h->h_dyn[0].nag;
  cudaStream_t q = h->stream;
  launch_dump_laminar(h->db, h->d_ci1, q);
  SPH_CUDA(cudaGetLastError());
  SPH_CUDA(cudaMemcpyAsync(flags, h->d_ci1, sizeof(int) * n, cudaMemcpyDefault, q));
  return cuda_status(cudaStreamSynchronize(q));
}

int sph_dump_renormalisation(SphHandle* h, double* b_gradp, double* b_divu) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || h->nsims != 1 || !h->any_c1) return SPH_ERR_INVALID_ARGUMENT;
  if (b_divu && !h->any_c1_divu) return SPH_ERR_INVALID_ARGUMENT;
  SPH_TRY(sync_dyn(h));
  int n = h->h_dyn[0].nag;
  double *dg = nullptr, *dd = nullptr;
  if (b_gradp) SPH_TRY(dalloc(&dg, (size_t)n * 9));
  if (b_divu && dalloc(&dd, (size_t)n * 9) != SPH_OK) { cudaFree(dg); return SPH_ERR_ALLOC; }
  cudaStream_t q = h->stream;
  launch_dump_renormalisation(h->db, dg, dd, q);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && dg) e = cudaMemcpyAsync(b_gradp, dg, sizeof(double) * 9 * (size_t)n, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess && dd) e = cudaMemcpyAsync(b_divu, dd, sizeof(double) * 9 * (size_t)n, cudaMemcpyDeviceToHost, q);
  if (e == cudaSuccess) e = cudaStreamSynchronize(q);
  cudaFree(dg);
  cudaFree(dd);
  return cuda_status(e);
}

// ---------------------------------------------------------------- autotuner
// Sizes the persistent grid of each kernel class on the live state: every
// candidate (1 to 32 blocks per SM) is timed over `reps` launches of a
// variant that leaves the state unchanged -- the rate-only momentum and
// continuity passes (their laminar-flag write is saved and restored), the
// neighbour-list and boundary passes (idempotent) -- and the fastest kept.
// The step graph is rebuilt with the choice.  grid_out[0..4] receives the
// chosen blocks of lists, momentum, continuity, boundary find, integrals,
// grid_out[5..6] the FP32c momentum and continuity loop shapes.

// Applies a launch configuration (sph_autotune's output, or a chosen one):
// blocks per kernel class (0 = the default) and the two pair-loop shapes.
int sph_set_launch_shape(SphHandle* h, const int32_t* shape) {
  DeviceGuard dev_guard_(h);
  if (!h || !shape) return SPH_ERR_INVALID_ARGUMENT;
  for (int c = 0; c < kGridClasses; ++c)
    if (shape[c] < 0) return SPH_ERR_INVALID_ARGUMENT;
  if (shape[kGridClasses] < 0 || shape[kGridClasses] > 2 || shape[kGridClasses + 1] < 0 ||
      shape[kGridClasses + 1] > 2)
    return SPH_ERR_INVALID_ARGUMENT;
  SPH_CUDA(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < kGridClasses; ++c) h->db.grid[c] = shape[c];
  h->db.mom_batch = shape[kGridClasses];
  h->db.con_batch = shape[kGridClasses + 1];
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  return SPH_OK;
}

int sph_autotune(SphHandle* h, int32_t reps, int32_t* grid_out) {
  DeviceGuard dev_guard_(h);
  NvtxRange range_("sph_autotune");
  if (!h || !h->uploaded || reps <= 0) return SPH_ERR_INVALID_ARGUMENT;
  cudaStream_t q = h->stream;
  DevBatch& b = h->db;
  const int mult[] = {1, 2, 4, 8, 16, 32};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) { cudaGetLastError(); return SPH_ERR_CUDA; }
  // the rate-only momentum pass rewrites the laminar flags: keep them
  SPH_CUDA(cudaMemcpyAsync(b.P.L2, b.P.L, (size_t)h->total_slots, cudaMemcpyDeviceToDevice, q));
  // with C1 the momentum (first step) and continuity passes complete and
  // invert the renormalisation matrices in place: keep them too
  const size_t nb_bytes = sizeof(double) * 9 * (size_t)h->total_slots;
  double *keep_g = nullptr, *keep_d = nullptr;
  cudaError_t e = cudaSuccess;
  if (h->any_c1) {
    e = cudaMallocAsync(&keep_g, nb_bytes, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(keep_g, b.P.BG, nb_bytes, cudaMemcpyDeviceToDevice, q);
  }
  if (e == cudaSuccess && h->any_c1_divu) {
    e = cudaMallocAsync(&keep_d, nb_bytes, q);
    if (e == cudaSuccess) e = cudaMemcpyAsync(keep_d, b.P.BD, nb_bytes, cudaMemcpyDeviceToDevice, q);
  }
  // the momentum and continuity pair loops come in two shapes (lean, or
  // several list entries' records loaded together), the FP32c loops in a
  // third (batched, two entries' terms on paired FP32 instructions): all
  // are timed
  const bool two_shapes = !h->any_c1;
  const int pair_shapes = h->precision == SPH_PREC_FP32C ? 3 : 2;
  int best_batch = b.mom_batch, best_cbatch = b.con_batch;
  for (int cls = 0; cls < kGridClasses && e == cudaSuccess; ++cls) {
    if (cls == kGridIntegrals && h->dim != 3) continue;
    float best = 1e30f;
    int best_g = 0;
    const int nshapes = (two_shapes && (cls == kGridMomentum || cls == kGridContinuity)) ? pair_shapes : 1;
    for (int cand = 0; cand < nshapes * 6; ++cand) {
      const int m = mult[cand % 6];
      if (nshapes > 1 && cls == kGridMomentum) b.mom_batch = cand / 6;
      if (nshapes > 1 && cls == kGridContinuity) b.con_batch = cand / 6;
      int g = b.sms * m;
      b.grid[cls] = g;
      auto run = [&]() {
        switch (cls) {
          case kGridLists: launch_neighbour_lists(b, q); break;
          case kGridMomentum: momentum_pass(h, false, q); break;
          case kGridContinuity: continuity_pass(h, false, q); break;
          default: launch_boundary(b, q); break;
        }
      };
      run();   // warm-up
      cudaEventRecord(e0, q);
      for (int r = 0; r < reps; ++r) run();
      cudaEventRecord(e1, q);
      e = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) break;
      if (ms < best) {
        best = ms;
        best_g = g;
        if (nshapes > 1 && cls == kGridMomentum) best_batch = b.mom_batch;
        if (nshapes > 1 && cls == kGridContinuity) best_cbatch = b.con_batch;
      }
    }
    b.grid[cls] = best_g;
    if (grid_out) grid_out[cls] = best_g;
    if (cls == kGridMomentum) b.mom_batch = best_batch;
    if (cls == kGridContinuity) b.con_batch = best_cbatch;
  }
  if (grid_out) {
    grid_out[kGridClasses] = b.mom_batch;
    grid_out[kGridClasses + 1] = b.con_batch;
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(b.P.L, b.P.L2, (size_t)h->total_slots, cudaMemcpyDeviceToDevice, q);
  if (e == cudaSuccess && keep_g) e = cudaMemcpyAsync(b.P.BG, keep_g, nb_bytes, cudaMemcpyDeviceToDevice, q);
  if (e == cudaSuccess && keep_d) e = cudaMemcpyAsync(b.P.BD, keep_d, nb_bytes, cudaMemcpyDeviceToDevice, q);
  if (keep_g) cudaFreeAsync(keep_g, q);
  if (keep_d) cudaFreeAsync(keep_d, q);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_status(e);
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  SPH_TRY(sync_dyn(h));
  return build_graph(h);
}

// ---------------------------------------------------------------- profiling
// Per-phase device time of nsteps un-graphed steps (CUDA events on the
// handle's stream; the replacement of the reference's start_and_stop timers,
// src/Post_processing/elapsed_time/start_and_stop.f90):
//   ms[0] momentum (RHS_momentum_equation + leapfrog + trajectories)
//   ms[1] OrdGrid1 (bin, removals, scan, place, rank/permute)
//   ms[2] ComputeBoundaryDataTab
//   ms[3] neighbour lists (CalcVarLength)
//   ms[4] continuity + Leapfrog_continuity + EoS
//   ms[5] time_step_duration closing
int sph_profile_phases(SphHandle* h, int32_t nsteps, double* ms) {
  DeviceGuard dev_guard_(h);
  if (!h || !h->uploaded || nsteps <= 0 || !ms) return SPH_ERR_INVALID_ARGUMENT;
  cudaEvent_t ev[7];
  for (int i = 0; i < 7; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) { cudaGetLastError(); return SPH_ERR_CUDA; }
  for (int i = 0; i < 6; ++i) ms[i] = 0.0;
  cudaStream_t q = h->stream;
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < nsteps && e == cudaSuccess; ++s) {
    cudaEventRecord(ev[0], q);
    momentum_pass(h, true, q);
    if (h->any_teta_v) launch_velocity_smoothing(h->db, true, h->precision == SPH_PREC_FP32C, q);
    cudaEventRecord(ev[1], q);
    sort_sequence(h, q);
    cudaEventRecord(ev[2], q);
    launch_boundary(h->db, q);
    cudaEventRecord(ev[3], q);
    lists_pass(h, q);
    cudaEventRecord(ev[4], q);
    continuity_pass(h, true, q);
    if (h->any_teta_p) launch_pressure_smoothing(h->db, h->precision == SPH_PREC_FP32C, q);
    cudaEventRecord(ev[5], q);
    launch_finalize(h->db, 1, q);
    cudaEventRecord(ev[6], q);
    e = cudaEventSynchronize(ev[6]);
    for (int i = 0; i < 6 && e == cudaSuccess; ++i) {
      float t = 0.f;
      e = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      ms[i] += t;
    }
  }
  for (int i = 0; i < 7; ++i) cudaEventDestroy(ev[i]);
  if (e != cudaSuccess) return cuda_status(e);
  return sync_dyn(h);
}

// Candidates tested and pairs accepted (incl. the particle itself) by the
// neighbour-list pass: c[0], c[1]; c[2..3] are reserved (zero).
int sph_get_counters(SphHandle* h, uint64_t* c, int32_t reset) {
  DeviceGuard dev_guard_(h);
  if (!h || !c) return SPH_ERR_INVALID_ARGUMENT;
  unsigned long long t[4];
  SPH_CUDA(cudaMemcpyAsync(t, h->d_counters, sizeof(t), cudaMemcpyDeviceToHost, h->stream));
  if (reset) SPH_CUDA(cudaMemsetAsync(h->d_counters, 0, sizeof(t), h->stream));
  SPH_CUDA(cudaStreamSynchronize(h->stream));
  for (int i = 0; i < 4; ++i) c[i] = t[i];
  return SPH_OK;
}

// Dense FP64 (fp32 = 0) or FP32 (fp32 = 1) FMA throughput of the current
// device (TFLOP/s): the arithmetic roofline of the pair passes.
int sph_measure_fma_peak(int32_t fp32, double* tflops) {
  if (!tflops) return SPH_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  double* sink = nullptr;
  int blocks = sms * 16;
  SPH_TRY(dalloc(&sink, blocks));
  cudaStream_t q;
  if (cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking) != cudaSuccess) { cudaFree(sink); cudaGetLastError(); return SPH_ERR_CUDA; }
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double flops = 0.0;
  for (int w = 0; w < 3; ++w) {
    if (fp32) launch_fp32_probe((float*)sink, blocks, q);
    else launch_fp64_probe(sink, blocks, q);
  }
  cudaEventRecord(a, q);
  for (int r = 0; r < 10; ++r) flops += fp32 ? launch_fp32_probe((float*)sink, blocks, q) : launch_fp64_probe(sink, blocks, q);
  cudaEventRecord(b, q);
  cudaError_t e = cudaEventSynchronize(b);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(q);
  cudaFree(sink);
  if (e != cudaSuccess) return cuda_status(e);
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SPH_OK;
}

int sph_measure_fp64_peak(double* tflops) { return sph_measure_fma_peak(0, tflops); }

// The kernels' exact division (div_rn) against the IEEE division on count
// generated operand pairs of the current device.
int sph_check_division(uint64_t count, uint64_t seed, uint64_t* mismatches, double* first_bad) {
  if (!mismatches) return SPH_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  unsigned long long* bad = nullptr;
  double* first = nullptr;
  SPH_TRY(dalloc(&bad, 2));
  if (dalloc(&first, 2) != SPH_OK) { cudaFree(bad); return SPH_ERR_ALLOC; }
  unsigned long long hb[2] = {0, 0};
  double hf[2] = {0.0, 0.0};
  cudaError_t e = cudaMemset(bad, 0, sizeof(hb));
  if (e == cudaSuccess) e = cudaMemset(first, 0, sizeof(hf));
  if (e == cudaSuccess) {
    launch_check_division(count, seed, bad, first, sms * 8, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(hb, bad, sizeof(hb), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(hf, first, sizeof(hf), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  cudaFree(first);
  if (e != cudaSuccess) return cuda_status(e);
  *mismatches = hb[0];
  if (first_bad) {
    first_bad[0] = hf[0];
    first_bad[1] = hf[1];
  }
  return SPH_OK;
}

}  // extern "C"
