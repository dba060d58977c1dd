// SPHERA hot-path ORACLE -- test infrastructure only.
//
// A CPU (FP64, OpenMP) restatement of the per-step SA-SPH particle path of
// SPHERA v10.0.0 (GiordanoAgateRSE/SPHERA, Fortran 90).  It exists to check
// the CUDA library and to time a CPU baseline; nothing in the product links
// or calls it.
//
// Parity status: PARITY UNPINNED by reference outputs.  The reference is
// Fortran only and no Fortran compiler exists on these machines, and the
// reference ships no tests, golden vectors or stored outputs.  The
// restatement is pinned instead by known-answer checks derived from the
// reference's own sources (the literal BoundIntegralTab2D table, the closed
// forms of IWro2dro/JdWsRn/WIntegr/J2Wro2, kernel normalisation, neighbour
// symmetry) and by an independent O(N^2) cross-check in the test suite.
//
// Layout follows the reference so the restatement stays auditable: an AoS
// particle array pg(1:nag) (1-based), Icont(1:nmax+1), NPartOrd(1:nag),
// materialised PartIntorno / PartKernel / rag lists of NMAXPARTJ slots per
// particle, BoundaryDataPointer(3,:) and BoundaryDataTab(:).
//
// Arithmetic is written in the reference's left-to-right evaluation order and
// compiled with -ffp-contract=off: the reference is built with gfortran -O2
// for baseline x86-64 (no FMA), src/Makefile:124.
//
// Scope: Domain%tipo = "semi" (SA-SPH), time_split = 1 (leapfrog), one
// liquid medium, all particles vel_type = "std", state = "flu"; ALE3,
// C1_BE, KTGF, DB-SPH, bodies off; wall zones "fixe" and
// "tapi" with slip_coefficient_mode = 1.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../include/sphera_b200.h"

namespace {

// Static_allocation_module.f90:27-77,142-150
constexpr double PIGRECO = 3.14159265358979e0;
constexpr double KERNELCONST3D = 1.0 / PIGRECO;
constexpr double KERNELCONST2D = 0.454728408833987e0;
constexpr double FI_INTERVAL = PIGRECO / 2.0;
constexpr double TETA_INTERVAL = PIGRECO + PIGRECO;
constexpr int FI_STEPS = 8;
constexpr int TETA_STEPS = 4 * FI_STEPS;
constexpr int BITrows = FI_STEPS * TETA_STEPS;
constexpr int INT_KERNELTABLE = 40;
constexpr int ktrows = INT_KERNELTABLE;
constexpr double max_positive_number = 3.4e+38;
// GI = 9.80665 is a default-REAL literal in Static_allocation_module.f90:72,
// so the double holds the single-precision rounding of 9.80665.
const double GI = (double)9.80665f;
constexpr int MAXCLOSEBOUNDSIDES = 4;
constexpr int LIMCLOSEBOUNDSIDES = 4;

// SA_SPH_module.f90:29-54.  The DATA values are default-REAL (E-format)
// literals: each double holds the single-precision rounding of the decimal.
const float BIT2D_LIT[22][6] = {
{-9.900000E-02f,6.916001E-01f,5.671769E-01f,1.614238E+00f,7.329450E-01f,8.813822E-01f},
{ 1.000000E-03f,6.820633E-01f,4.993001E-01f,1.426603E+00f,7.142813E-01f,7.123606E-01f},
{ 1.010000E-01f,6.725266E-01f,4.314232E-01f,1.238968E+00f,6.956176E-01f,5.433391E-01f},
{ 2.010000E-01f,6.452481E-01f,3.653947E-01f,1.057834E+00f,6.492812E-01f,4.085521E-01f},
{ 3.010000E-01f,6.025034E-01f,3.028878E-01f,8.871524E-01f,5.851007E-01f,3.020341E-01f},
{ 4.010000E-01f,5.473293E-01f,2.453079E-01f,7.296175E-01f,5.106232E-01f,2.189841E-01f},
{ 5.010000E-01f,4.832434E-01f,1.937172E-01f,5.872117E-01f,4.319031E-01f,1.553082E-01f},
{ 6.010000E-01f,4.139976E-01f,1.488267E-01f,4.612826E-01f,3.538107E-01f,1.074685E-01f},
{ 7.010000E-01f,3.434138E-01f,1.109601E-01f,3.526284E-01f,2.802530E-01f,7.237218E-02f},
{ 8.010000E-01f,2.751568E-01f,8.006434E-02f,2.615428E-01f,2.142205E-01f,4.732315E-02f},
{ 9.010000E-01f,2.125249E-01f,5.573915E-02f,1.877770E-01f,1.577964E-01f,2.998003E-02f},
{ 1.001000E+00f,1.581202E-01f,3.728314E-02f,1.304301E-01f,1.120873E-01f,1.834320E-02f},
{ 1.101000E+00f,1.131765E-01f,2.379696E-02f,8.756287E-02f,7.679627E-02f,1.076657E-02f},
{ 1.201000E+00f,7.737532E-02f,1.434262E-02f,5.638309E-02f,5.038764E-02f,5.995379E-03f},
{ 1.301000E+00f,4.995510E-02f,8.042085E-03f,3.441001E-02f,3.129118E-02f,3.118804E-03f},
{ 1.401000E+00f,2.994721E-02f,4.104289E-03f,1.956203E-02f,1.807987E-02f,1.482120E-03f},
{ 1.501000E+00f,1.623613E-02f,1.842642E-03f,1.008625E-02f,9.464607E-03f,6.216584E-04f},
{ 1.601000E+00f,7.615461E-03f,6.873181E-04f,4.510624E-03f,4.293336E-03f,2.172841E-04f},
{ 1.701000E+00f,2.842820E-03f,1.913104E-04f,1.609094E-03f,1.552266E-03f,5.682598E-05f},
{ 1.801000E+00f,6.998383E-04f,3.120105E-05f,3.793334E-04f,3.706037E-04f,8.729655E-06f},
{ 1.901000E+00f,6.214235E-05f,1.372448E-06f,3.231651E-05f,3.195398E-05f,3.625237E-07f},
{ 2.001000E+00f,0.000000E+00f,0.000000E+00f,0.000000E+00f,0.000000E+00f,0.000000E+00f}};
constexpr double DELTAX_BIT = 0.1;

// TyParticle subset (Hybrid_allocation_module.f90:159-387).
struct Particle {
  double coord[3], vel[3], var[3], acc[3], velass[3];
  double dens, pres, mass, dden, kin_visc;
  int cella, kodvel, koddens, laminar_flag;
  double Bg[3][3], Bd[3][3];   // B_ren_gradp, B_ren_divu: Bg[i][j] = B(i+1,j+1)
};

struct Face {           // TyBoundaryFace
  int nodes;
  int name[6];
  double GX[6][3];
  double LX[6][2];
  double T[3][3];       // T[row][col] = T(row+1,col+1)
  double Area;
  int stretch;          // 1-based zone
  double velocity[3];
};

struct Side {           // TyBoundarySide
  int vertex[2];        // 1-based vertex ids
  int stretch;
  double length;
  double T[3][3];
  double RN[3][3];
  double velocity[3];
  double angle;
  int previous_side;    // 1-based, 0 = none
};

struct ConvexEdge {     // TyBoundaryConvexEdge
  int face[2];          // 1-based face ids
  double GX1[3];        // node(1)%GX
  double component[3];
  double length;
};

struct BDT {            // TyBoundaryData
  int CloBoNum;
  double LocXYZ[3];
  double BoundaryIntegral[8];
  double IntGiWrRdV[3][3];
};

struct Oracle {
  SphParams prm;
  int dim;              // 2 or 3
  int ncord;
  // Domain / derived (ReadInput.f90:198-205, Gest_Input.f90:266-289)
  double h, doubleh, squareh, square_doubleh, unosuh, unosusquareh, eta, eta2;
  double coefke, coefkacl, celerita;
  int NMAXPARTJ;
  // Grid (CreaGrid.f90)
  double extr[3][2], dcd[3];
  int ncd[3], nmax;
  // particles, 1-based
  int nag;
  std::vector<Particle> pg;
  std::vector<int> Icont, NPartOrd;
  std::vector<int> nPartIntorno, PartIntorno;
  std::vector<double> PartKernel;  // [4][slot] stored as slot*4+k
  std::vector<double> rag;         // slot*3+k
  int EpOrdGrid = 0;
  int truncated = 0;
  // zones
  std::vector<SphZone> zones;
  std::vector<double> vert;        // 1-based: vert[3*(id-1)+k]
  // 3D faces
  std::vector<Face> faces;         // index nf-1
  std::vector<int> BFaceList;      // 1-based face ids
  std::vector<ConvexEdge> BoundaryConvexEdge;
  std::vector<int> GCBFptr_n, GCBFptr_s;  // per cell (1-based)
  std::vector<int> GCBFVector;     // 1-based positions
  double kerneltab[ktrows + 1][5];
  double ktdelta;
  double BIT[BITrows][7];
  // 2D sides
  std::vector<Side> sides;
  double BIT2D[22][6];
  // boundary data
  std::vector<int> BDP;            // 3 per particle: BDP[3*(npi-1)+k]
  std::vector<BDT> BDTab;          // slot (MAXCLOSE*(npi-1)+icbf)-1
  int maxcb;                       // MAXCLOSEBOUNDFACES or MAXCLOSEBOUNDSIDES
  int Ncbf_Max = 0;
  int fatal = 0;
  // time
  double dt = 0, dt_average = 0, simulation_time = 0, dtvel = 0;
  int on_going_time_step = -999;
  int nthreads = 1;
  // body force used by RHS_momentum_equation: prm.grav plus the lateral tank
  // forcing (an extension of the library, absent from the reference)
  double geff[3] = {0, 0, 0};
};

// Sine of the forcing phase, the same sequence of IEEE operations as the
// library's device function: reduction by the nearest multiple of 2 pi,
// folding into [-pi/2, pi/2], Taylor series to r^23 in nested form.
static double forcing_sin(double x) {
  const double two_pi = 6.283185307179586, pi = 3.141592653589793, half_pi = 1.5707963267948966;
  double k = std::nearbyint(x / two_pi);
  double r = x - k * two_pi;
  if (r > half_pi) r = pi - r;
  else if (r < -half_pi) r = -pi - r;
  double r2 = r * r;
  double t = 1.0;
  for (int n = 22; n >= 2; n -= 2) t = 1.0 - r2 / (double)(n * (n + 1)) * t;
  return r * t;
}

// geff at simulation time t: grav + A w^2 sin(w t) along x, w = 2 pi / T,
// for a tank moving as x = A sin(w t); equal to grav when A = 0.
static void set_body_force(Oracle& o, double t) {
  for (int d = 0; d < 3; ++d) o.geff[d] = o.prm.grav[d];
  if (o.prm.forcing_amplitude != 0.0) {
    double w = 6.283185307179586 / o.prm.forcing_period;
    double aw2 = o.prm.forcing_amplitude * w * w;
    o.geff[0] = o.prm.grav[0] + aw2 * forcing_sin(w * t);
  }
}

inline double sq3(double a) { return (a * a) * a; }

// ------------------------------------------------------------------------
// Grid helpers
// ------------------------------------------------------------------------

// CreaGrid.f90:51-74
void CreaGrid(Oracle& o) {
  double epsi = 0.01 * o.prm.dx;
  double dextr[3];
  for (int d = 0; d < 3; ++d) {
    o.extr[d][0] = o.prm.domain_lo[d] - o.doubleh - epsi;
    o.extr[d][1] = o.prm.domain_hi[d] + o.doubleh + epsi;
    dextr[d] = o.extr[d][1] - o.extr[d][0];
    o.ncd[d] = (int)std::lround(dextr[d] / o.doubleh);   // NINT
    o.dcd[d] = dextr[d] / o.ncd[d];
  }
  if (o.dim == 2) o.ncd[1] = 1;
  o.nmax = o.ncd[0] * o.ncd[1] * o.ncd[2];
}

// CellNumber.f90:53-59
inline int CellNumber(const Oracle& o, int i, int j, int k) {
  if (i < 1 || i > o.ncd[0] || j < 1 || j > o.ncd[1] || k < 1 || k > o.ncd[2]) return 0;
  return ((k - 1) * o.ncd[1] + (j - 1)) * o.ncd[0] + i;
}

// ParticleCellNumber.f90:52-62
inline int ParticleCellNumber(const Oracle& o, const double* coord) {
  double xp = coord[0] - o.extr[0][0];
  double yp = coord[1] - o.extr[1][0];
  double zp = coord[2] - o.extr[2][0];
  int i = (int)std::ceil(xp / o.dcd[0]);
  int k = (int)std::ceil(zp / o.dcd[2]);
  int j = (o.dim == 3) ? (int)std::ceil(yp / o.dcd[1]) : 1;
  return CellNumber(o, i, j, k);
}

// CellIndices.f90:51-63
inline int CellIndices(const Oracle& o, int nc, int& i, int& j, int& k) {
  int ni = o.ncd[0], nj = o.ncd[1];
  int nucellsij = ni * nj;
  k = (nc - 1) / nucellsij + 1;
  int ncij = nc - nucellsij * (k - 1);
  j = (ncij - 1) / ni + 1;
  i = ncij - ni * (j - 1);
  return ncij;
}

// OrdGrid1.f90:50-105 (fluid particles part)
void OrdGrid1(Oracle& o) {
  std::vector<int> cnt(o.nmax + 1, 0);
  std::fill(o.Icont.begin(), o.Icont.end(), 0);
  int npi = 0;
  while (o.nag > 0 && npi < o.nag) {
    npi = npi + 1;
    Particle& p = o.pg[npi];
    int ncel = ParticleCellNumber(o, p.coord);
    if (ncel <= 0 || ncel > o.nmax) {
      // out of grid: swap with the last particle, OrdGrid1.f90:71-82
      o.EpOrdGrid += 1;
      o.pg[npi] = o.pg[o.nag];
      o.pg[o.nag] = Particle{};
      o.nag -= 1;
      npi -= 1;
    } else {
      o.Icont[ncel] += 1;
      p.cella = ncel;
      o.Icont[o.nmax + 1] += 1;
    }
  }
  for (int i = o.nmax; i >= 1; --i) o.Icont[i] = o.Icont[i + 1] - o.Icont[i];
  for (int i = 1; i <= o.nmax + 1; ++i) o.Icont[i] += 1;
  for (npi = 1; npi <= o.nag; ++npi) {
    int ncel = o.pg[npi].cella;
    if (ncel == 0) continue;
    o.NPartOrd[o.Icont[ncel] + cnt[ncel]] = npi;
    cnt[ncel] += 1;
  }
}

// CalcVarLength.f90:133-269, SA-SPH branch (C1_BE, KTGF, bodies off)
// grad_W_sub.f90:52-91 (3D): gradient of the beta-spline (kernel_ID 1) or
// anti-cluster (kernel_ID 2) kernel at r_vec; PIGRECO as
// Static_allocation_module.f90:50.
static void grad_W_sub(const Oracle& o, int kernel_ID, const double* r_vec, double* grad_W) {
  const double PIGRECO = 3.14159265358979;
  grad_W[0] = grad_W[1] = grad_W[2] = 0.0;
  double abs_r = std::sqrt(r_vec[0] * r_vec[0] + r_vec[1] * r_vec[1] + r_vec[2] * r_vec[2]);
  if (abs_r < o.h * 1.0e-6) return;
  double q = abs_r / o.h;
  double h3 = o.h * o.h * o.h;
  double dW = 0.0;
  if (kernel_ID == 1) {
    if (q <= 1.0) dW = 1.0 / (PIGRECO * h3) * (9.0 / 4.0 * (q * q) - 3.0 * q);
    else if (q >= 2.0) dW = 0.0;
    else dW = -(3.0 / (4.0 * PIGRECO * h3) * ((2.0 - q) * (2.0 - q)));
  } else {
    if (q <= 2.0) dW = -(3.0 * ((2.0 - q) * (2.0 - q)) * (15.0 / (64.0 * PIGRECO * h3)));
  }
  for (int k = 0; k < 3; ++k) grad_W[k] = dW / o.h * r_vec[k] / abs_r;
  if (o.dim == 2) {   // grad_W_sub.f90:79-88 (SPACE_2D)
    for (int k = 0; k < 3; ++k)
      grad_W[k] = (kernel_ID == 1) ? grad_W[k] * o.h * 10.0 / 7.0 : grad_W[k] * o.h * 4.0 / 3.0;
  }
}

// Matrix_Inversion_3x3.f90:50-74 inside B_ren_gradp_inversion.f90 /
// B_ren_divu_inversion.f90:58-75: the inverse when |det| >= thresh, else -I.
static void B_ren_inversion(double B[3][3], double thresh) {
  double det = B[0][0] * B[1][1] * B[2][2] + B[1][0] * B[2][1] * B[0][2] + B[2][0] * B[0][1] * B[1][2] -
               B[0][0] * B[2][1] * B[1][2] - B[2][0] * B[1][1] * B[0][2] - B[1][0] * B[0][1] * B[2][2];
  if (std::fabs(det) >= thresh) {
    double inv[3][3];
    inv[0][0] = B[1][1] * B[2][2] - B[1][2] * B[2][1];
    inv[0][1] = B[0][2] * B[2][1] - B[0][1] * B[2][2];
    inv[0][2] = B[0][1] * B[1][2] - B[0][2] * B[1][1];
    inv[1][0] = B[1][2] * B[2][0] - B[1][0] * B[2][2];
    inv[1][1] = B[0][0] * B[2][2] - B[0][2] * B[2][0];
    inv[1][2] = B[0][2] * B[1][0] - B[0][0] * B[1][2];
    inv[2][0] = B[1][0] * B[2][1] - B[1][1] * B[2][0];
    inv[2][1] = B[0][1] * B[2][0] - B[0][0] * B[2][1];
    inv[2][2] = B[0][0] * B[1][1] - B[0][1] * B[1][0];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[i][j] = inv[i][j] / det;
  } else {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) B[i][j] = 0.0;
    B[0][0] = B[1][1] = B[2][2] = -1.0;
  }
}

// v = -(B v) (MatrixProduct.f90:55-63, then the sign of the callers).
static void B_renormalise(const double B[3][3], double* v) {
  double a[3];
  for (int i = 0; i < 3; ++i) {
    double sum = 0.0;
    for (int k = 0; k < 3; ++k) sum = sum + B[i][k] * v[k];
    a[i] = sum;
  }
  for (int i = 0; i < 3; ++i) v[i] = -a[i];
}

// T (IntGiWrRdV T^T): the SA-SPH frontier's contribution to the
// renormalisation matrices (AddBoundaryContributions_to_ME3D.f90:172-187,
// AddBoundaryContribution_to_CE3D.f90:93-112).
static void frontier_B(const Face& f, const BDT& e, double out[3][3]) {
  double Tt[3][3], m2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Tt[i][j] = f.T[j][i];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k) sum = sum + e.IntGiWrRdV[i][k] * Tt[k][j];
      m2[i][j] = sum;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k) sum = sum + f.T[i][k] * m2[k][j];
      out[i][j] = sum;
    }
}

void CalcVarLength(Oracle& o) {
  const double ke_coef = o.coefke / o.h;
  const double kacl_coef = o.coefkacl / o.h;
  const int NM = o.NMAXPARTJ;
  std::fill(o.nPartIntorno.begin(), o.nPartIntorno.end(), 0);
  int trunc_count = 0;
#pragma omp parallel for schedule(static) num_threads(o.nthreads) reduction(+:trunc_count)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& pi = o.pg[npi];
    int nceli = pi.cella;
    if (nceli == 0) continue;
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) pi.Bg[a][c] = pi.Bd[a][c] = 0.0;   // CalcVarLength.f90:181-182
    int igridi, jgridi, kgridi;
    CellIndices(o, nceli, igridi, jgridi, kgridi);
    int jgrid1 = jgridi - (o.ncord - 2);
    int jgrid2 = jgridi + (o.ncord - 2);
    bool warned = false;
    for (int jrang = jgrid1; jrang <= jgrid2; ++jrang)
      for (int irang = igridi - 1; irang <= igridi + 1; ++irang)
        for (int krang = kgridi - 1; krang <= kgridi + 1; ++krang) {
          int ncelj = CellNumber(o, irang, jrang, krang);
          if (ncelj == 0) continue;
          for (int mm = o.Icont[ncelj]; mm <= o.Icont[ncelj + 1] - 1; ++mm) {
            if (o.nPartIntorno[npi] >= NM) { warned = true; continue; }
            int npj = o.NPartOrd[mm];
            const Particle& pj = o.pg[npj];
            double rt[3];
            rt[0] = pi.coord[0] - pj.coord[0];
            rt[1] = pi.coord[1] - pj.coord[1];
            rt[2] = pi.coord[2] - pj.coord[2];
            double rijtemp = rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2];
            if (rijtemp > o.square_doubleh) continue;
            o.nPartIntorno[npi] += 1;
            long npartint = (long)(npi - 1) * NM + o.nPartIntorno[npi];
            o.PartIntorno[npartint] = npj;
            double rijtemp2 = rijtemp;
            rijtemp = std::sqrt(rijtemp);
            double rij_su_h = rijtemp / o.h;
            double rij_su_h_quad = rijtemp2 / o.squareh;
            int index_rij_su_h = (int)rij_su_h;
            double denom = 1.0 / (rijtemp + o.eta);
            double* rg = &o.rag[npartint * 3];
            rg[0] = rt[0]; rg[1] = rt[1]; rg[2] = rt[2];
            double* pk = &o.PartKernel[npartint * 4];
            pk[0] = pk[1] = pk[2] = pk[3] = 0.0;
            if (index_rij_su_h >= 2) continue;
            double gradmod = -(2.0 * rij_su_h) + 1.5 * rij_su_h_quad;
            double gradmodwacl = -12.0 - 3.0 * rij_su_h_quad + 12.0 * rij_su_h;
            double wu = 0.666666667 + rij_su_h_quad * (rij_su_h * 0.5 - 1.0);
            if (index_rij_su_h > 0) {
              gradmod = -gradmod + rij_su_h_quad - 2.0;
              wu = (2.0 - rij_su_h) * (2.0 - rij_su_h) * (2.0 - rij_su_h) * 0.166666666667;
            }
            gradmod = gradmod * ke_coef;
            gradmodwacl = gradmodwacl * kacl_coef;
            pk[0] = gradmod * denom;
            pk[1] = pk[0] / (rijtemp2 + o.eta2);
            pk[2] = gradmodwacl * denom;
            pk[3] = wu * o.coefke;
            if (o.prm.c1_be) {
              // CalcVarLength.f90:285-324: the renormalisation matrices
              double r_vec[3] = {-rt[0], -rt[1], -rt[2]}, gW[3], gWo[3];
              const double dxj[3] = {pj.coord[0] - pi.coord[0], pj.coord[1] - pi.coord[1], pj.coord[2] - pi.coord[2]};
              grad_W_sub(o, 2, r_vec, gW);
              for (int k = 0; k < 3; ++k) gWo[k] = gW[k] * pj.mass / pj.dens;
              for (int c = 0; c < 3; ++c)
                for (int k = 0; k < 3; ++k) pi.Bg[k][c] = pi.Bg[k][c] + dxj[c] * gWo[k];
              if (o.prm.c1_divu) {
                grad_W_sub(o, 1, r_vec, gW);
                for (int k = 0; k < 3; ++k) gWo[k] = gW[k] * pj.mass / pj.dens;
                for (int c = 0; c < 3; ++c)
                  for (int k = 0; k < 3; ++k) pi.Bd[k][c] = pi.Bd[k][c] + dxj[c] * gWo[k];
              }
            }
          }
        }
    if (warned) trunc_count += 1;
  }
  o.truncated += trunc_count;
}

// ------------------------------------------------------------------------
// SA-SPH 3D geometry and tables
// ------------------------------------------------------------------------

// Vector_Product.f90
inline void Vector_Product(const double* u, const double* v, double* w) {
  const int iseg[3] = {1, 2, 0};
  for (int i = 0; i < 3; ++i) {
    int j = iseg[i], k = iseg[j];
    w[i] = u[j] * v[k] - u[k] * v[j];
  }
}

// DefineLocalSystemVersors.f90 (3D face frame, local node coordinates)
void DefineLocalSystemVersors(Oracle& o, Face& f) {
  const int nindex[2][3] = {{1, 2, 3}, {1, 3, 4}};
  int nnodes = f.nodes;
  int sidek = nnodes - 2;
  for (int n = 0; n < nnodes; ++n)
    for (int i = 0; i < 3; ++i) f.GX[n][i] = o.vert[3 * (f.name[n] - 1) + i];
  double U1[3], U2[3], RR[3], W12[3], nn[3], ss[3];
  for (int i = 0; i < 3; ++i) {
    U1[i] = f.GX[nindex[sidek - 1][0] - 1][i] - f.GX[nindex[sidek - 1][2] - 1][i];
    U2[i] = f.GX[nindex[sidek - 1][1] - 1][i] - f.GX[nindex[sidek - 1][2] - 1][i];
  }
  double U1len = std::sqrt(U1[0] * U1[0] + U1[1] * U1[1] + U1[2] * U1[2]);
  for (int i = 0; i < 3; ++i) RR[i] = U1[i] / U1len;
  Vector_Product(U1, U2, W12);
  double W12len = std::sqrt(W12[0] * W12[0] + W12[1] * W12[1] + W12[2] * W12[2]);
  f.Area = W12len / (double)(float)(3 - sidek);
  for (int i = 0; i < 3; ++i) nn[i] = W12[i] / W12len;
  Vector_Product(nn, RR, ss);
  for (int i = 0; i < 3; ++i) { f.T[i][0] = RR[i]; f.T[i][1] = ss[i]; f.T[i][2] = nn[i]; }
  int refnode = nnodes;
  for (int n = 1; n <= nnodes - 1; ++n)
    for (int i = 0; i < 2; ++i) {
      double LocX = 0.0;
      for (int j = 0; j < 3; ++j)
        LocX = LocX + f.T[j][i] * (f.GX[n - 1][j] - f.GX[refnode - 1][j]);
      f.LX[n - 1][i] = LocX;
    }
  f.LX[refnode - 1][0] = 0.0;
  f.LX[refnode - 1][1] = 0.0;
}

// GridCellBoundaryFacesIntersections3D.f90:89-210
void GridCellBoundaryFacesIntersections3D(Oracle& o) {
  o.GCBFptr_n.assign(o.nmax + 1, 0);
  o.GCBFptr_s.assign(o.nmax + 1, 0);
  o.GCBFVector.assign(1, 0);
  for (int nc = 1; nc <= o.nmax; ++nc) {
    int i, j, k;
    CellIndices(o, nc, i, j, k);
    double CellXYZ[3][2];
    int idx[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
      CellXYZ[d][0] = o.extr[d][0] + o.dcd[d] * (idx[d] - 1);
      CellXYZ[d][1] = o.extr[d][0] + o.dcd[d] * idx[d];
    }
    double CellNodeXYZ[8][3];
    int nv = 0;
    for (int ii = 0; ii < 2; ++ii)
      for (int jj = 0; jj < 2; ++jj)
        for (int kk = 0; kk < 2; ++kk) {
          CellNodeXYZ[nv][0] = CellXYZ[0][ii];
          CellNodeXYZ[nv][1] = CellXYZ[1][jj];
          CellNodeXYZ[nv][2] = CellXYZ[2][kk];
          nv++;
        }
    int count = 0;
    for (size_t kf = 0; kf < o.BFaceList.size(); ++kf) {
      const Face& f = o.faces[o.BFaceList[kf] - 1];
      int nodes = f.nodes;
      bool Found = true;
      for (int sd = 0; sd < 3 && Found; ++sd) {
        int sc[5] = {0, 0, 0, 0, 0};   // Signcount(-2:2)
        for (int no = 0; no < nodes; ++no) {
          double X = f.GX[no][sd];
          if (X < CellXYZ[sd][0]) sc[0]++;
          else if (X == CellXYZ[sd][0]) sc[1]++;
          else if (X < CellXYZ[sd][1]) sc[2]++;
          else if (X == CellXYZ[sd][1]) sc[3]++;
          else if (X > CellXYZ[sd][1]) sc[4]++;
        }
        if ((sc[0] + sc[1]) == nodes && !(sc[1] == nodes)) Found = false;
        else if ((sc[4] + sc[3]) == nodes && !(sc[3] == nodes)) Found = false;
      }
      if (!Found) continue;
      int sc[3] = {0, 0, 0};
      for (nv = 0; nv < 8; ++nv) {
        double zita = 0.0;
        for (int sd = 0; sd < 3; ++sd) {
          double d = CellNodeXYZ[nv][sd] - f.GX[nodes - 1][sd];
          zita = zita + f.T[sd][2] * d;
        }
        if (zita < 0.0) sc[0]++;
        else if (zita == 0.0) sc[1]++;
        else sc[2]++;
      }
      if ((sc[0] + sc[1]) == 8 && !(sc[1] == 4)) Found = false;
      else if ((sc[2] + sc[1]) == 8 && !(sc[1] == 4)) Found = false;
      if (Found) {
        if (count == 0) o.GCBFptr_s[nc] = (int)o.GCBFVector.size();
        o.GCBFVector.push_back(o.BFaceList[kf]);
        count++;
      }
    }
    o.GCBFptr_n[nc] = count;
  }
}

// ComputeBoundaryIntegralTab.f90:61-86
void ComputeBoundaryIntegralTab(Oracle& o) {
  double delta_fi = FI_INTERVAL / FI_STEPS;
  double delta_fimz = 0.5 * delta_fi;
  double duesendelta_fimz = 2.0 * std::sin(delta_fimz);
  double delta_teta = TETA_INTERVAL / TETA_STEPS;
  int points = 0;
  double fi = -0.5 * delta_fi;
  for (int i = 1; i <= FI_STEPS; ++i) {
    fi = fi + delta_fi;
    double teta = -0.5 * delta_teta;
    double zp = -(o.doubleh * std::cos(fi));
    for (int j = 1; j <= TETA_STEPS; ++j) {
      teta = teta + delta_teta;
      double xp = o.doubleh * std::sin(fi) * std::cos(teta);
      double yp = o.doubleh * std::sin(fi) * std::sin(teta);
      double delta_alpha = delta_teta * duesendelta_fimz * std::sin(fi);
      o.BIT[points][0] = xp;
      o.BIT[points][1] = yp;
      o.BIT[points][2] = zp;
      o.BIT[points][3] = delta_alpha;
      o.BIT[points][4] = xp / o.doubleh;
      o.BIT[points][5] = yp / o.doubleh;
      o.BIT[points][6] = zp / o.doubleh;
      points++;
    }
  }
}

// IWro2dro.f90:60-74
double IWro2dro(double ro) {
  const double a1 = 0.333333333333333, a2 = 0.3, a3 = 0.125, a4 = 0.25;
  const double b1 = 0.0625, b2 = 0.025, b3 = 4.16666666666667e-03;
  if (ro >= 0.0 && ro < 1.0) {
    double ro2 = ro * ro;
    double ro3 = ro2 * ro;
    double I1 = (a1 - a2 * ro2 + a3 * ro3) * ro3;
    return KERNELCONST3D * (a4 - I1);
  } else if (ro >= 1.0 && ro < 2.0) {
    double ro2 = ro * ro;
    double duemro = 2.0 - ro;
    double duemro2 = duemro * duemro;
    double duemro4 = duemro2 * duemro2;
    double I2 = -(b1 * ro2 + b2 * duemro * ro + b3 * duemro2) * duemro4;
    return KERNELCONST3D * (-I2);
  }
  return 0.0;
}

// JdWsRn.f90 (kernel = 1, beta-spline)
double JdWsRn(double ro, int n) {
  const double KS3D = 0.31830989;
  double ro2 = ro * ro, ro3 = ro2 * ro, ro4 = ro2 * ro2, ro5 = ro4 * ro;
  double J = 0.0;
  switch (n) {
    case 0:
      if (ro >= 0.0 && ro < 1.0) J = -1.0 + (1.5 - 0.75 * ro) * ro2;
      else if (ro >= 1.0 && ro < 2.0) { double d = 2.0 - ro; J = -0.25 * d * d * d; }
      break;
    case 1:
      if (ro >= 0.0 && ro < 1.0) J = -0.75 + (1.0 - 0.5625 * ro) * ro3;
      else if (ro >= 1.0 && ro < 2.0) J = -1.0 + (1.5 - 1.0 * ro + 0.1875 * ro2) * ro2;
      break;
    case 2:
      if (ro >= 0.0 && ro < 1.0) J = -0.7 + (0.75 - 0.45 * ro) * ro4;
      else if (ro >= 1.0 && ro < 2.0) J = -0.8 + (1.0 - 0.75 * ro + 0.15 * ro2) * ro3;
      break;
    case 3:
      if (ro >= 0.0 && ro < 1.0) J = -0.75 + (0.6 - 0.375 * ro) * ro5;
      else if (ro >= 1.0 && ro < 2.0) J = -0.8 + (0.75 - 0.6 * ro + 0.125 * ro2) * ro4;
      break;
    default: J = 0.0;
  }
  return J * KS3D;
}

// ComputeKernelTable.f90:58-71
void ComputeKernelTable(Oracle& o) {
  o.ktdelta = 2.0 / INT_KERNELTABLE;
  for (int nr = 0; nr <= ktrows; ++nr) {
    double rob = o.ktdelta * nr;
    o.kerneltab[nr][0] = rob;
    o.kerneltab[nr][1] = IWro2dro(rob);
    o.kerneltab[nr][2] = JdWsRn(rob, 1) * o.unosusquareh;
    o.kerneltab[nr][3] = JdWsRn(rob, 2) * o.unosuh;
    o.kerneltab[nr][4] = JdWsRn(rob, 3);
  }
}

// InterpolateTable.f90:58-82 (columns 1..4)
void InterpolateTable(const Oracle& o, double xval, double* ivalue) {
  double deltaX = o.ktdelta;
  double xval0 = o.kerneltab[0][0];
  int nr0 = (int)((xval - xval0) / deltaX);
  if (nr0 <= 0) {
    for (int c = 0; c < 4; ++c) ivalue[c] = o.kerneltab[0][c + 1];
  } else if (nr0 >= ktrows) {
    for (int c = 0; c < 4; ++c) ivalue[c] = o.kerneltab[ktrows][c + 1];
  } else {
    int nr1 = nr0 + 1;
    double csi = (xval - o.kerneltab[nr0][0]) / deltaX;
    for (int c = 0; c < 4; ++c)
      ivalue[c] = o.kerneltab[nr0][c + 1] + csi * (o.kerneltab[nr1][c + 1] - o.kerneltab[nr0][c + 1]);
  }
}

// LocalNormalCoordinates.f90:59-87
void LocalNormalCoordinates(const Face& f, const double* PX, double* csi) {
  const int iseg[3] = {2, 3, 1};
  const int mainod[2][3] = {{1, 2, 3}, {1, 3, 4}};
  int fkod = f.nodes - 2;
  double DueArea = (double)(3 - fkod) * f.Area;
  double UsuDueArea = 1.0 / DueArea;
  for (int ii = 1; ii <= 2; ++ii) {
    int jj = iseg[ii - 1];
    int kk = iseg[jj - 1];
    double xj = f.LX[mainod[fkod - 1][jj - 1] - 1][0];
    double yj = f.LX[mainod[fkod - 1][jj - 1] - 1][1];
    double xk = f.LX[mainod[fkod - 1][kk - 1] - 1][0];
    double yk = f.LX[mainod[fkod - 1][kk - 1] - 1][1];
    double AA = xj * yk - xk * yj;
    double BB = yj - yk;
    double CC = xk - xj;
    csi[ii - 1] = (AA + BB * PX[0] + CC * PX[1]) * UsuDueArea;
  }
  csi[2] = 1.0 - (csi[0] + csi[1]);
}

// IsPointInternal.f90:54-72
bool IsPointInternal(int fk, const double* csi) {
  if (fk == 1) {
    for (int ii = 0; ii < 3; ++ii) { if (csi[ii] < 0.0) return false; if (csi[ii] > 1.0) return false; }
    return true;
  } else if (fk == 2) {
    for (int ii = 0; ii < 2; ++ii) { if (csi[ii] < 0.0) return false; if (csi[ii] > 1.0) return false; }
    return true;
  }
  return false;
}

// FindCloseBoundaryFaces3D.f90:79-188 (zones fixe/tapi)
int FindCloseBoundaryFaces3D(Oracle& o, int npi, int& Ncbf, int* Clobface, double (*LocX)[3]) {
  const Particle& p = o.pg[npi];
  Ncbf = 0;
  int nc = ParticleCellNumber(o, p.coord);
  if (nc <= 0) return 0;
  int ic, jc, kc;
  CellIndices(o, nc, ic, jc, kc);
  for (int i = ic - 1; i <= ic + 1; ++i)
    for (int j = jc - 1; j <= jc + 1; ++j)
      for (int k = kc - 1; k <= kc + 1; ++k) {
        int ncl = CellNumber(o, i, j, k);
        if (ncl == 0) continue;
        int nfpercell = o.GCBFptr_n[ncl];
        if (nfpercell <= 0) continue;
        int flpini = o.GCBFptr_s[ncl];
        for (int flp = flpini; flp <= flpini + nfpercell - 1; ++flp) {
          int intbf = o.GCBFVector[flp];
          double pinmin = 0.0, pinmax = o.doubleh;
          bool thereis = false;
          for (int q = 0; q < Ncbf; ++q) if (Clobface[q] == intbf) thereis = true;
          if (thereis) continue;
          const Face& f = o.faces[intbf - 1];
          double PXLoc[3];
          for (int sdi = 0; sdi < 3; ++sdi) {
            PXLoc[sdi] = 0.0;
            for (int sdj = 0; sdj < 3; ++sdj)
              PXLoc[sdi] = PXLoc[sdi] + f.T[sdj][sdi] * (p.coord[sdj] - f.GX[f.nodes - 1][sdj]);
          }
          double pin = PXLoc[2];
          if (pin >= pinmin && pin < pinmax) {
            Ncbf = Ncbf + 1;
            if (Ncbf <= o.maxcb) {
              Clobface[Ncbf - 1] = intbf;
              LocX[Ncbf - 1][2] = pin;
            } else {
              return SPH_ERR_CLOSE_FACES;
            }
          }
        }
      }
  for (int icbf = 0; icbf < Ncbf; ++icbf) {
    const Face& f = o.faces[Clobface[icbf] - 1];
    for (int sdi = 0; sdi < 2; ++sdi) {
      LocX[icbf][sdi] = 0.0;
      for (int sdj = 0; sdj < 3; ++sdj)
        LocX[icbf][sdi] = LocX[icbf][sdi] + f.T[sdj][sdi] * (p.coord[sdj] - f.GX[f.nodes - 1][sdj]);
    }
  }
  return 0;
}

// ComputeBoundaryVolumeIntegrals_P0.f90:81-155
void ComputeBoundaryVolumeIntegrals_P0(const Oracle& o, const Face& f, const double* LocXin, BDT& e) {
  const double eps = 0.05;
  double IntWdV = 0, IntdWrm1dV = 0, IntGWZrm1dV = 0;
  double IntGWdV[3] = {0, 0, 0};
  double IntGWrRdV[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double JW3ro2dA = 0, JdW3ro1dA = 0, JdW3ro2dA = 0, JdW3ro3dA = 0;
  double zpmin = eps * o.h;
  double LocPi[3] = {LocXin[0], LocXin[1], LocXin[2]};
  int fkod = f.nodes - 2;
  if (!(LocPi[2] < 0.0)) {
    if (LocPi[2] < zpmin) LocPi[2] = zpmin;
    double robpre = 2.1;
    for (int ipk = 0; ipk < BITrows; ++ipk) {
      double LocPj[3];
      for (int d = 0; d < 3; ++d) LocPj[d] = LocPi[d] + o.BIT[ipk][d];
      if (LocPj[2] <= 0) {
        double tsegnato = LocPi[2] / (LocPi[2] - LocPj[2]);
        double PXLoc[3];
        for (int d = 0; d < 3; ++d) PXLoc[d] = LocPi[d] + (LocPj[d] - LocPi[d]) * tsegnato;
        PXLoc[2] = 0.0;
        double csi[3];
        LocalNormalCoordinates(f, PXLoc, csi);
        if (IsPointInternal(fkod, csi)) {
          double PiPxdist = 0.0;
          for (int SD = 0; SD < 3; ++SD) {
            double dd = PXLoc[SD] - LocPi[SD];
            PiPxdist = PiPxdist + dd * dd;
          }
          PiPxdist = std::sqrt(PiPxdist);
          double delta_alpha = o.BIT[ipk][3];
          double rob = PiPxdist / o.h;
          if (std::fabs(rob - robpre) > 1.0e-3) {
            double iv[4];
            InterpolateTable(o, rob, iv);
            JW3ro2dA = iv[0] * delta_alpha;
            JdW3ro1dA = iv[1] * delta_alpha;
            JdW3ro2dA = iv[2] * delta_alpha;
            JdW3ro3dA = iv[3] * delta_alpha;
            robpre = rob;
          }
          double RL[3] = {o.BIT[ipk][4], o.BIT[ipk][5], o.BIT[ipk][6]};
          double RZ = RL[2];
          double RZ2 = RZ * RZ;
          IntWdV = IntWdV + JW3ro2dA;
          IntdWrm1dV = IntdWrm1dV + JdW3ro1dA;
          IntGWZrm1dV = IntGWZrm1dV + RZ2 * JdW3ro1dA;
          for (int SD = 0; SD < 3; ++SD) {
            IntGWdV[SD] = IntGWdV[SD] + RL[SD] * JdW3ro2dA;
            for (int sdj = SD; sdj < 3; ++sdj)
              IntGWrRdV[SD][sdj] = IntGWrRdV[SD][sdj] + RL[SD] * RL[sdj] * JdW3ro3dA;
          }
        }
      }
    }
    IntGWrRdV[1][0] = IntGWrRdV[0][1];
    IntGWrRdV[2][0] = IntGWrRdV[0][2];
    IntGWrRdV[2][1] = IntGWrRdV[1][2];
    if (LocPi[2] == zpmin) {
      double PXLoc[3] = {LocPi[0], LocPi[1], 0.0};
      double csi[3];
      LocalNormalCoordinates(f, PXLoc, csi);
      IntWdV = IsPointInternal(fkod, csi) ? 0.5 : 0.0;
    }
  }
  e.BoundaryIntegral[0] = 0.0;
  e.BoundaryIntegral[1] = IntWdV;
  e.BoundaryIntegral[2] = IntdWrm1dV;
  e.BoundaryIntegral[3] = IntGWdV[0];
  e.BoundaryIntegral[4] = IntGWdV[1];
  e.BoundaryIntegral[5] = IntGWdV[2];
  e.BoundaryIntegral[6] = IntGWZrm1dV;
  e.BoundaryIntegral[7] = 0.0;
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) e.IntGiWrRdV[a][b] = IntGWrRdV[a][b];
}

// ComputeBoundaryDataTab_3D.f90:67-105
int ComputeBoundaryDataTab_3D(Oracle& o) {
  std::fill(o.BDP.begin(), o.BDP.end(), 0);
  int status = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    if (o.pg[npi].cella <= 0) continue;
    int Ncbf;
    std::vector<int> Clob(o.maxcb + 1, 0);
    std::vector<double> LocXv(3 * (o.maxcb + 1), 0.0);
    double (*LocX)[3] = reinterpret_cast<double (*)[3]>(LocXv.data());
    int st = FindCloseBoundaryFaces3D(o, npi, Ncbf, Clob.data(), LocX);
    if (st) {
#pragma omp critical(ora_status)
      { if (!status) status = st; }
      continue;
    }
    int* bdp = &o.BDP[3 * (npi - 1)];
    if (Ncbf == 0) { bdp[0] = bdp[1] = bdp[2] = 0; continue; }
    bdp[0] = Ncbf;
    bdp[1] = 0;
    long ibdt = (long)o.maxcb * (npi - 1);
    bdp[2] = (int)(ibdt + 1);
    for (int icbf = 0; icbf < Ncbf; ++icbf) {
      BDT& e = o.BDTab[ibdt + icbf];
      const Face& f = o.faces[Clob[icbf] - 1];
      ComputeBoundaryVolumeIntegrals_P0(o, f, LocX[icbf], e);
      e.CloBoNum = Clob[icbf];
      for (int d = 0; d < 3; ++d) e.LocXYZ[d] = LocX[icbf][d];
    }
  }
  return status;
}

// ------------------------------------------------------------------------
// SA-SPH 2D
// ------------------------------------------------------------------------

// w.f90:48-57
double w_kernel(double r, double h, double coef) {
  const double a1 = 0.666666667;
  double s = r / h, q;
  if (s <= 1.0) q = a1 + s * s * (s * 0.5 - 1.0);
  else if (s >= 2.0) q = 0.0;
  else { double dms = 2.0 - s; q = dms * dms * dms / 6.0; }
  return q * coef;
}

// WIntegr.f90:57-74
double WIntegr(double ri, double hh) {
  const double a = 0.5, a2 = -0.375, a3 = 0.15, aa = -0.125, aa1 = 0.05, b = 0.35;
  double ro = ri / hh;
  if (0.0 <= ro && ro < 1.0) {
    double ro2 = ro * ro, ro3 = ro2 * ro;
    double W1 = (a + a2 * ro2 + a3 * ro3) * ro2;
    return KERNELCONST2D * (b - W1);
  } else if (1.0 <= ro && ro < 2.0) {
    double q1 = 2.0 - ro, q2 = q1 * q1, q4 = q2 * q2;
    double W2 = (aa + aa1 * q1) * q4;
    return -KERNELCONST2D * W2;
  }
  return 0.0;
}

// J2Wro2.f90:50-63
double J2Wro2(double ro) {
  const double a1 = 0.00833333333333333, a2 = 0.26666666666666667;
  double ro2 = ro * ro, ro3 = ro2 * ro;
  if (0.0 <= ro && ro < 1.0)
    return KERNELCONST2D * (0.25 - (a1 * (40.0 - 36.0 * ro2 + 15.0 * ro3) * ro3));
  else if (1.0 <= ro && ro < 2.0)
    return KERNELCONST2D * (a2 - (a1 * (80.0 - 90.0 * ro + 36.0 * ro2 - 5.0 * ro3) * ro3));
  return 0.0;
}

// DefineBoundarySideGeometry2D.f90 + BoundaryMassForceMatrix2D.f90 +
// DefineBoundarySideRelativeAngles2D.f90 (fixe/tapi zones)
void DefineBoundarySideGeometry2D(Oracle& o) {
  for (auto& s : o.sides) {
    const double* V1 = &o.vert[3 * (s.vertex[0] - 1)];
    const double* V2 = &o.vert[3 * (s.vertex[1] - 1)];
    double Dx = V2[0] - V1[0];
    double Dz = V2[2] - V1[2];
    double L = std::sqrt(Dx * Dx + Dz * Dz);
    double sx = Dx / L, sz = Dz / L;
    std::memset(s.T, 0, sizeof(s.T));
    s.length = L;
    s.T[0][0] = sx;
    s.T[2][0] = sz;
    s.T[0][2] = -sz;
    s.T[2][2] = sx;
    double FiS = 1.0, FiN = 1.0;
    std::memset(s.RN, 0, sizeof(s.RN));
    s.RN[0][0] = FiS * s.T[0][0] * s.T[0][0] + FiN * s.T[2][0] * s.T[2][0];
    s.RN[0][2] = (FiS - FiN) * s.T[0][0] * s.T[2][0];
    s.RN[2][0] = s.RN[0][2];
    s.RN[2][2] = FiS * s.T[2][0] * s.T[2][0] + FiN * s.T[0][0] * s.T[0][0];
    const SphZone& z = o.zones[s.stretch - 1];
    for (int d = 0; d < 3; ++d) s.velocity[d] = (z.type == SPH_ZONE_TAPI) ? z.velocity[d] : 0.0;
  }
  int ns = (int)o.sides.size();
  for (int isi = 0; isi < ns; ++isi) {
    int ksi = 0;
    for (int jsi = 0; jsi < ns; ++jsi)
      if (o.sides[jsi].vertex[1] == o.sides[isi].vertex[0]) { ksi = jsi + 1; break; }
    o.sides[isi].angle = 0.0;
    if (ksi > 0) {
      const double (*Tm)[3] = o.sides[isi].T;
      const double (*PT)[3] = o.sides[ksi - 1].T;
      double sinangle = PT[0][0] * Tm[2][0] - PT[2][0] * Tm[0][0];
      double cosangle = PT[0][0] * Tm[0][0] + PT[2][0] * Tm[2][0];
      o.sides[isi].angle = std::atan2(sinangle, cosangle);
    }
    o.sides[isi].previous_side = ksi;
  }
}

// InterpolateBoundaryIntegrals2D.f90:61-69
void InterpolateBoundaryIntegrals2D(const Oracle& o, int Ncols, const int* Colmn, double xx, double* Func) {
  if (xx < o.BIT2D[0][0]) xx = o.BIT2D[0][0];
  int ii = (int)((xx - o.BIT2D[0][0]) / DELTAX_BIT) + 1;
  double xi = o.BIT2D[ii - 1][0];
  for (int nc = 0; nc < Ncols; ++nc) {
    int jj = Colmn[nc];
    double fi = o.BIT2D[ii - 1][jj];
    double fip1 = o.BIT2D[ii][jj];
    Func[nc] = fi + (fip1 - fi) * (xx - xi) / DELTAX_BIT;
  }
}

// FindCloseBoundarySides2D.f90:78-208 (no "sour" zones)
int FindCloseBoundarySides2D(const Oracle& o, int npi, int& Ncbs, int* Cloboside, double (*LocXY)[2]) {
  const Particle& p = o.pg[npi];
  Ncbs = 0;
  double Plocal[2] = {p.coord[0], p.coord[2]};
  double ypmin = -o.doubleh, ypmax = o.doubleh;
  int ns = (int)o.sides.size();
  for (int isi = 1; isi <= ns; ++isi) {
    const Side& s = o.sides[isi - 1];
    const double* V1 = &o.vert[3 * (s.vertex[0] - 1)];
    double P1P[2] = {Plocal[0] - V1[0], Plocal[1] - V1[2]};
    double sss[2] = {s.T[0][0], s.T[2][0]};
    double nnn[2] = {s.T[0][2], s.T[2][2]};
    double sidel = s.length;
    double xp = P1P[0] * sss[0] + P1P[1] * sss[1];
    double yp = P1P[0] * nnn[0] + P1P[1] * nnn[1];
    double xpmin = -o.doubleh, xpmax = sidel + o.doubleh;
    if ((xpmin < xp && xp < xpmax) && (ypmin < yp && yp < ypmax)) {
      double ypmx = 0, ypmn = 0;
      if (xp < 0.0) {
        double xpq = xp * xp;
        ypmx = std::sqrt(o.square_doubleh - xpq);
        ypmn = -ypmx;
      } else if (xp <= sidel) {
        ypmx = ypmax;
        ypmn = ypmin;
      } else if (xp < xpmax) {
        double Lmxpq = (sidel - xp) * (sidel - xp);
        ypmx = std::sqrt(o.square_doubleh - Lmxpq);
        ypmn = -ypmx;
      }
      if (ypmn < yp && yp < ypmx) {
        Ncbs = Ncbs + 1;
        if (Ncbs > MAXCLOSEBOUNDSIDES) return SPH_ERR_CLOSE_SIDES;
        Cloboside[Ncbs - 1] = isi;
        LocXY[Ncbs - 1][0] = xp;
        LocXY[Ncbs - 1][1] = yp;
      }
    }
  }
  if (Ncbs > LIMCLOSEBOUNDSIDES) return 809;
  if (Ncbs == 2) {
    int iside1 = Cloboside[0], iside2 = Cloboside[1];
    if (o.sides[iside1 - 1].previous_side == iside2) {
      LocXY[1][0] = o.sides[iside2 - 1].length - LocXY[1][0];
    } else if (o.sides[iside2 - 1].previous_side == iside1) {
      LocXY[0][0] = o.sides[iside1 - 1].length - LocXY[0][0];
    }
  }
  return 0;
}

// SelectCloseBoundarySides2D.f90:72-121 (fixe/tapi branch)
void SelectCloseBoundarySides2D(int Ncbs, const int* Cloboside, const double (*LocXY)[2],
                                int& IntNcbs, int* Intboside, double (*IntLocXY)[2]) {
  IntNcbs = 0;
  for (int icbs = 0; icbs < Ncbs; ++icbs) {
    if (LocXY[icbs][1] > 0.0) {
      Intboside[IntNcbs] = Cloboside[icbs];
      IntLocXY[IntNcbs][0] = LocXY[icbs][0];
      IntLocXY[IntNcbs][1] = LocXY[icbs][1];
      IntNcbs++;
    }
  }
}

// FindBoundaryIntersection2D.f90:61-92
void FindBoundaryIntersection2D(const Oracle& o, int icbs, const int* Cloboside, const double (*LocXY)[2],
                                double& xpmin, double& xpmax, double& interlen) {
  double eps = 0.01;
  double minlen = eps * o.h;
  interlen = 0.0;
  double xpi = LocXY[icbs][0], ypi = LocXY[icbs][1];
  if (ypi < 0.0) ypi = 0.0;
  double ypiq = ypi * ypi;
  double halfchord = std::sqrt(o.square_doubleh - ypiq);
  double XA = xpi - halfchord, XB = xpi + halfchord;
  double bsidelen = o.sides[Cloboside[icbs] - 1].length;
  xpmin = 0.0;
  if (XA > xpmin) xpmin = XA;
  xpmax = bsidelen;
  if (XB < xpmax) xpmax = XB;
  interlen = xpmax - xpmin;
  if (interlen <= minlen) interlen = 0.0;
}

// ComputeSurfaceIntegral_WdS2D.f90:57-83
double ComputeSurfaceIntegral_WdS2D(const Oracle& o, int icbs, const double (*LocXY)[2], double xpmin, double interlen) {
  const int ndivrif = 2;
  double SIntWds = 0.0;
  double dsrif = o.h / ndivrif;
  if (interlen > 0.0) {
    double xpi = LocXY[icbs][0], ypi = LocXY[icbs][1];
    if (ypi < 0.0) ypi = 0.0;
    double ypiq = ypi * ypi;
    int ndiv = (int)(interlen / dsrif + 0.5);
    if (ndiv < ndivrif) ndiv = ndivrif;
    double deltas = interlen / ndiv;
    double xpip = xpmin - 0.5 * deltas;
    for (int ipt = 1; ipt <= ndiv; ++ipt) {
      xpip = xpip + deltas;
      double dxpip = xpip - xpi;
      double risq = dxpip * dxpip + ypiq;
      double ris = std::sqrt(risq);
      double Wds = w_kernel(ris, o.h, o.coefke) * deltas;
      SIntWds = SIntWds + Wds;
    }
  }
  return SIntWds;
}

// BoundaryVolumeIntegrals2D.f90
void BoundaryVolumeIntegrals2D(const Oracle& o, int icbs, const double (*LocXY)[2], double xpmin, double xpmax,
                               double interlen, double& IntWdV, double* IntDpWdV) {
  const int Nalfadiv = 10;
  const double eps = 0.05;
  double dalfarif = PIGRECO / Nalfadiv;
  IntWdV = 0.0;
  IntDpWdV[0] = IntDpWdV[1] = 0.0;
  if (interlen <= 0.0) return;
  double yplimite = eps * o.h;
  double xpi = LocXY[icbs][0], ypi = LocXY[icbs][1];
  if (ypi < yplimite) ypi = yplimite;
  double csiPA = xpmin - xpi, csiPB = xpmax - xpi;
  double alfaA = std::atan2(csiPA, ypi), alfaB = std::atan2(csiPB, ypi);
  double Intalfa = alfaB - alfaA;
  int ndiv = (int)(Intalfa / dalfarif + 0.5);
  if (ndiv < 1) ndiv = 1;
  double dalfa = Intalfa / ndiv;
  double alfa_k = alfaA - 0.5 * dalfa;
  for (int k = 1; k <= ndiv; ++k) {
    alfa_k = alfa_k + dalfa;
    double sinalfa = std::sin(alfa_k), cosalfa = std::cos(alfa_k);
    double rb = ypi / cosalfa;
    double rob = rb / o.h;
    double mult = o.h * J2Wro2(rob) * dalfa;
    IntDpWdV[0] = IntDpWdV[0] + sinalfa * mult;
    IntDpWdV[1] = IntDpWdV[1] - cosalfa * mult;
    IntWdV = IntWdV + WIntegr(rb, o.h) * dalfa;
  }
  if (ypi == yplimite) IntWdV = 0.5;
}

// ComputeVolumeIntegral_WdV2D.f90
int ComputeVolumeIntegral_WdV2D(const Oracle& o, int icbs, int Ncbslocal, const int* Cloboside,
                                const double (*LocXY)[2], double xpmin, double xpmax, double interlen,
                                double& VIntWdV) {
  const int Nalfadiv = 10;
  const double eps = 0.05;
  double dalfarif = PIGRECO / Nalfadiv;
  VIntWdV = 0.0;
  if (interlen <= 0.0) return 0;
  double yplimite = eps * o.h;
  double xpi = LocXY[icbs][0], ypi = LocXY[icbs][1];
  if (ypi >= yplimite) {
    double csiPA = xpmin - xpi, etaPA = ypi, csiPB = xpmax - xpi, etaPB = ypi;
    double alfaA = std::atan2(csiPA, etaPA), alfaB = std::atan2(csiPB, etaPB);
    double Intalfa = alfaB - alfaA;
    int ndiv = (int)(Intalfa / dalfarif + 0.5);
    if (ndiv < 2) ndiv = 2;
    double dalfa = Intalfa / ndiv;
    double alfa = alfaA - 0.5 * dalfa;
    for (int ipt = 1; ipt <= ndiv; ++ipt) {
      alfa = alfa + dalfa;
      double tanalfa = std::tan(alfa);
      double ris = ypi * std::sqrt(1.0 + tanalfa * tanalfa);
      VIntWdV = VIntWdV + WIntegr(ris, o.h) * dalfa;
    }
  } else if (ypi < yplimite && Ncbslocal == 1) {
    VIntWdV = (xpmin >= xpi && xpi <= xpmax) ? 0.5 : 0.0;
  } else if (ypi < yplimite && Ncbslocal == 2) {
    int jcbs = Ncbslocal + 1 - (icbs + 1);
    double ypj = LocXY[jcbs - 1][1];
    if (ypj <= yplimite) {
      double angle = 0.0;
      if (o.sides[Cloboside[0] - 1].previous_side == Cloboside[1]) angle = o.sides[Cloboside[0] - 1].angle;
      else if (o.sides[Cloboside[1] - 1].previous_side == Cloboside[0]) angle = o.sides[Cloboside[1] - 1].angle;
      else return 804;
      VIntWdV = 0.5 * (angle + PIGRECO) / (2.0 * PIGRECO);
    } else {
      VIntWdV = (xpmin >= xpi && xpi <= xpmax) ? 0.5 : 0.0;
    }
  }
  return 0;
}

// ComputeBoundaryDataTab_2D.f90:70-157
int ComputeBoundaryDataTab_2D(Oracle& o) {
  std::fill(o.BDP.begin(), o.BDP.end(), 0);
  int status = 0;
#pragma omp parallel for schedule(dynamic, 256) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    if (o.pg[npi].cella <= 0) continue;
    int Ncbs, Clob[MAXCLOSEBOUNDSIDES + 1];
    double LocXY[MAXCLOSEBOUNDSIDES + 1][2];
    int st = FindCloseBoundarySides2D(o, npi, Ncbs, Clob, LocXY);
    if (st) {
#pragma omp critical(ora_status)
      { if (!status) status = st; }
      continue;
    }
    if (Ncbs <= 0) continue;
    int IntNcbs, Intb[MAXCLOSEBOUNDSIDES];
    double IntLocXY[MAXCLOSEBOUNDSIDES][2];
    SelectCloseBoundarySides2D(Ncbs, Clob, LocXY, IntNcbs, Intb, IntLocXY);
    if (IntNcbs <= 0) continue;
    int* bdp = &o.BDP[3 * (npi - 1)];
    bdp[0] = Ncbs;
    bdp[1] = IntNcbs;
    long ibdt = (long)MAXCLOSEBOUNDSIDES * (npi - 1);
    bdp[2] = (int)(ibdt + 1);
    for (int icbs = 0; icbs < IntNcbs; ++icbs) {
      BDT& e = o.BDTab[ibdt + icbs];
      e.CloBoNum = Intb[icbs];
      e.LocXYZ[0] = IntLocXY[icbs][0];
      e.LocXYZ[1] = IntLocXY[icbs][1];
      e.LocXYZ[2] = 0.0;
      std::memset(e.IntGiWrRdV, 0, sizeof(e.IntGiWrRdV));
      double Func[5] = {0, 0, 0, 0, 0};
      if (IntNcbs == 2) {
        double xpmin, xpmax, interlen;
        FindBoundaryIntersection2D(o, icbs, Intb, IntLocXY, xpmin, xpmax, interlen);
        double IntWdS = ComputeSurfaceIntegral_WdS2D(o, icbs, IntLocXY, xpmin, interlen);
        double IntWdV, IntDpWdV[2], IntWdV1;
        BoundaryVolumeIntegrals2D(o, icbs, IntLocXY, xpmin, xpmax, interlen, IntWdV, IntDpWdV);
        int s2 = ComputeVolumeIntegral_WdV2D(o, icbs, IntNcbs, Intb, IntLocXY, xpmin, xpmax, interlen, IntWdV1);
        if (s2) {
#pragma omp critical(ora_status)
          { if (!status) status = s2; }
        }
        const int Colmn[3] = {3, 4, 5};
        double deltai = IntLocXY[icbs][1] / o.h;
        InterpolateBoundaryIntegrals2D(o, 3, Colmn, deltai, Func);
        e.BoundaryIntegral[0] = IntWdS;
        e.BoundaryIntegral[1] = IntWdV;
        e.BoundaryIntegral[2] = IntWdV1;
        e.BoundaryIntegral[3] = IntDpWdV[0];
        e.BoundaryIntegral[4] = IntDpWdV[1];
        e.BoundaryIntegral[5] = Func[0] / o.squareh;
        e.BoundaryIntegral[6] = Func[1] / o.squareh;
        e.BoundaryIntegral[7] = Func[2] / o.squareh;
      } else if (IntNcbs == 1) {
        const int Colmn[5] = {1, 2, 3, 4, 5};
        double deltai = IntLocXY[icbs][1] / o.h;
        InterpolateBoundaryIntegrals2D(o, 5, Colmn, deltai, Func);
        double IntWdS = Func[0] / o.h;
        double IntWdV = Func[1];
        e.BoundaryIntegral[0] = IntWdS;
        e.BoundaryIntegral[1] = IntWdV;
        e.BoundaryIntegral[2] = IntWdV;
        e.BoundaryIntegral[3] = 0.0;
        e.BoundaryIntegral[4] = 0.0;
        e.BoundaryIntegral[5] = Func[2] / o.squareh;
        e.BoundaryIntegral[6] = Func[3] / o.squareh;
        e.BoundaryIntegral[7] = Func[4] / o.squareh;
      }
    }
  }
  return status;
}

// ------------------------------------------------------------------------
// Continuity
// ------------------------------------------------------------------------

// AddBoundaryContribution_to_CE3D.f90:82-169 (C1_BE and ALE3 off)
void AddBoundaryContribution_to_CE3D(Oracle& o, int npi, int Ncbf, double* gu, double* gv, double* gw) {
  Particle& p = o.pg[npi];
  int ibdt = o.BDP[3 * (npi - 1) + 2];
  for (int icbf = 1; icbf <= Ncbf; ++icbf) {
    const BDT& e = o.BDTab[ibdt + icbf - 2];
    const Face& f = o.faces[e.CloBoNum - 1];
    if (e.LocXYZ[2] > 0.0) {
      if (o.prm.c1_be) {   // AddBoundaryContribution_to_CE3D.f90:93-112
        double m[3][3];
        frontier_B(f, e, m);
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c) {
            if (o.prm.c1_divu) p.Bd[a][c] = p.Bd[a][c] + m[a][c];
            p.Bg[a][c] = p.Bg[a][c] + m[a][c];
          }
      }
      double aux2[3], n[3], dvel[3], av[3];
      for (int d = 0; d < 3; ++d) aux2[d] = 2.0 * (f.velocity[d] - p.var[d]);
      for (int d = 0; d < 3; ++d) n[d] = f.T[d][2];
      double dp = 0.0;
      for (int d = 0; d < 3; ++d) dp = dp + aux2[d] * n[d];
      for (int d = 0; d < 3; ++d) dvel[d] = dp * n[d];
      for (int i = 0; i < 3; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s = s + f.T[i][k] * e.BoundaryIntegral[3 + k];
        av[i] = s;
      }
      for (int d = 0; d < 3; ++d) {
        gu[d] = gu[d] - dvel[0] * av[d];
        gv[d] = gv[d] - dvel[1] * av[d];
        gw[d] = gw[d] - dvel[2] * av[d];
      }
    }
  }
}

// AddBoundaryContribution_to_CE2D.f90:73-147 (ALE3 off)
void AddBoundaryContribution_to_CE2D(Oracle& o, int npi, int IntNcbs, double* gu, double* gw) {
  Particle& p = o.pg[npi];
  const int acix[2] = {0, 2};
  int ibdt = o.BDP[3 * (npi - 1) + 2];
  for (int icbs = 1; icbs <= IntNcbs; ++icbs) {
    const BDT& e = o.BDTab[ibdt + icbs - 2];
    const Side& s = o.sides[e.CloBoNum - 1];
    const SphZone& z = o.zones[s.stretch - 1];
    if (o.prm.c1_be) {   // AddBoundaryContribution_to_CE2D.f90:81-94: -RN IntWdV
      const double IntWdV = e.BoundaryIntegral[2];
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) {
          const double aux = -s.RN[a][c] * IntWdV;
          if (o.prm.c1_divu) p.Bd[a][c] = p.Bd[a][c] + aux;
          p.Bg[a][c] = p.Bg[a][c] + aux;
        }
    }
    double IntWdS = e.BoundaryIntegral[0];
    double dvel[2];
    if (z.type == SPH_ZONE_FIXE) {
      for (int pd = 0; pd < 2; ++pd) dvel[pd] = 2.0 * (-p.var[acix[pd]]);
    } else {
      for (int pd = 0; pd < 2; ++pd) dvel[pd] = 2.0 * (s.velocity[acix[pd]] - p.var[acix[pd]]);
    }
    for (int ii = 0; ii < 2; ++ii) {
      gu[acix[ii]] = gu[acix[ii]] - dvel[0] * s.T[acix[ii]][2] * IntWdS;
      gw[acix[ii]] = gw[acix[ii]] - dvel[1] * s.T[acix[ii]][2] * IntWdS;
    }
  }
}

// SASPH_continuity.f90:89-169 (C1_BE, ALE3 off)
void SASPH_continuity(Oracle& o, int npi, int& Ncbf_Max_local) {
  Particle& p = o.pg[npi];
  double gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
  bool active;
  if (o.dim == 3) {
    int Ncbf = o.BDP[3 * (npi - 1)];
    active = Ncbf > 0;
    if (active) {
      Ncbf_Max_local = std::max(Ncbf_Max_local, Ncbf);
      AddBoundaryContribution_to_CE3D(o, npi, Ncbf, gu, gv, gw);
    }
  } else {
    int Ncbs = o.BDP[3 * (npi - 1)], IntNcbs = o.BDP[3 * (npi - 1) + 1];
    active = Ncbs > 0 && IntNcbs > 0;
    if (active) AddBoundaryContribution_to_CE2D(o, npi, IntNcbs, gu, gw);
  }
  if (o.prm.c1_be) {   // SASPH_continuity.f90:112-119
    if (o.prm.c1_divu) B_ren_inversion(p.Bd, o.prm.invb_det_thresh);
    B_ren_inversion(p.Bg, o.prm.invb_det_thresh);
  }
  if (active && o.prm.c1_be && o.prm.c1_divu) {   // SASPH_continuity.f90:126-140
    B_renormalise(p.Bd, gu);
    if (o.dim == 3) B_renormalise(p.Bd, gv);
    B_renormalise(p.Bd, gw);
  }
  if (active && p.koddens == 0)
    p.dden = p.dden - p.dens * (gu[0] + gv[1] + gw[2]);
}

// Continuity_Equation.f90:90-249 (liquid, C1/ALE3 off, all neighbours std)
void Continuity_Equation(Oracle& o, int npi) {
  Particle& p = o.pg[npi];
  if (p.cella <= 0) return;
  if (o.prm.c1_be && o.prm.c1_divu) {
    // Continuity_Equation.f90:119-126,201-217: the whole velocity-gradient
    // vectors, renormalised with B_ren_divu
    double v1[3] = {0, 0, 0}, v2[3] = {0, 0, 0}, v3[3] = {0, 0, 0};
    for (int contj = 1; contj <= o.nPartIntorno[npi]; ++contj) {
      long npartint = (long)(npi - 1) * o.NMAXPARTJ + contj;
      const Particle& q = o.pg[o.PartIntorno[npartint]];
      double rhoi = p.dens, rhoj = q.dens, amassj = q.mass;
      double dvar[3] = {q.var[0] - p.var[0], q.var[1] - p.var[1], q.var[2] - p.var[2]};
      const double* rg = &o.rag[npartint * 3];
      double c = rhoi * (amassj / rhoj) * o.PartKernel[npartint * 4];
      for (int k = 0; k < 3; ++k) {
        v1[k] = v1[k] + c * dvar[0] * rg[k];
        if (o.dim == 3) v2[k] = v2[k] + c * dvar[1] * rg[k];
        v3[k] = v3[k] + c * dvar[2] * rg[k];
      }
    }
    B_renormalise(p.Bd, v1);
    if (o.dim == 3) B_renormalise(p.Bd, v2);
    B_renormalise(p.Bd, v3);
    p.dden = p.dden - (v1[0] + v2[1] + v3[2]);
    return;
  }
  double a1 = 0.0, a2 = 0.0, a3 = 0.0;
  const int NM = o.NMAXPARTJ;
  for (int contj = 1; contj <= o.nPartIntorno[npi]; ++contj) {
    long npartint = (long)(npi - 1) * NM + contj;
    int npj = o.PartIntorno[npartint];
    const Particle& q = o.pg[npj];
    double rhoi = p.dens, rhoj = q.dens, amassj = q.mass;
    double dvar[3] = {q.var[0] - p.var[0], q.var[1] - p.var[1], q.var[2] - p.var[2]};
    const double* rg = &o.rag[npartint * 3];
    double PK1 = o.PartKernel[npartint * 4];
    double c = rhoi * (amassj / rhoj) * PK1;
    a1 = a1 + c * dvar[0] * rg[0];
    if (o.dim == 3) a2 = a2 + c * dvar[1] * rg[1];
    a3 = a3 + c * dvar[2] * rg[2];
  }
  if (o.dim == 3) p.dden = p.dden - (a1 + a2 + a3);
  else p.dden = p.dden - (a1 + a3);
}

// ------------------------------------------------------------------------
// Momentum
// ------------------------------------------------------------------------

// AddBoundaryContributions_to_ME3D.f90:105-336 (fixe/tapi, mode 1, C1/ALE3 off)
void AddBoundaryContributions_to_ME3D(Oracle& o, int npi, int Ncbf, double* tpres, double* tdiss, double* tvisc) {
  Particle& p = o.pg[npi];
  const bool c1_first = o.prm.c1_be && o.on_going_time_step == 1;
  double vi[3] = {p.var[0], p.var[1], p.var[2]};
  double ALEt[3] = {0, 0, 0}, gradpt[3] = {0, 0, 0}, VMon[3] = {0, 0, 0}, VShear[3] = {0, 0, 0};
  for (int icbf = 1; icbf <= Ncbf; ++icbf) {
    const BDT& e = o.BDTab[o.BDP[3 * (npi - 1) + 2] + icbf - 2];
    const Face& f = o.faces[e.CloBoNum - 1];
    const SphZone& z = o.zones[f.stretch - 1];
    double nn[3] = {f.T[0][2], f.T[1][2], f.T[2][2]};
    if (!(e.LocXYZ[2] > 0.0)) continue;
    double dvn = 0.0, dvij[3];
    for (int SD = 0; SD < 3; ++SD) {
      dvij[SD] = 2.0 * (vi[SD] - f.velocity[SD]);
      dvn = dvn + f.T[SD][2] * dvij[SD];
    }
    double gl[3];
    for (int SD = 0; SD < 3; ++SD) {
      gl[SD] = 0.0;
      for (int sdj = 0; sdj < 3; ++sdj) gl[SD] = gl[SD] + f.T[sdj][SD] * o.geff[sdj];
    }
    double loc[3], glob[3];
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + e.IntGiWrRdV[i][k] * gl[k];
      loc[i] = s;
    }
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + f.T[i][k] * loc[k];
      glob[i] = s;
    }
    for (int d = 0; d < 3; ++d) gradpt[d] = gradpt[d] + glob[d];
    double aloc[3], aglob[3];
    for (int k = 0; k < 3; ++k) aloc[k] = 2.0 * p.pres / p.dens * e.BoundaryIntegral[3 + k];
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s = s + f.T[i][k] * aloc[k];
      aglob[i] = s;
    }
    for (int d = 0; d < 3; ++d) ALEt[d] = ALEt[d] + aglob[d];
    if (c1_first) {
      double m[3][3];
      frontier_B(f, e, m);
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) p.Bg[a][c] = p.Bg[a][c] + m[a][c];
    }
    double IntGWZrm1dV = e.BoundaryIntegral[6];
    double IntdWrm1dV = e.BoundaryIntegral[2];
    double alfaMon = o.prm.alfa_mon;
    if (alfaMon > 0.0) {
      double Monvisc = alfaMon * o.celerita * o.h;
      double Mmult = -(Monvisc * dvn * IntGWZrm1dV);
      for (int d = 0; d < 3; ++d) VMon[d] = VMon[d] + Mmult * nn[d];
    }
    double slip_coefficient = z.bc_shear_stress_input;
    double cinvisci = p.kin_visc;
    if (cinvisci > 0.0) {
      if (p.laminar_flag == 1 || !z.laminar_no_slip_check) {
        double cinviscmult = cinvisci * IntdWrm1dV * slip_coefficient;
        for (int d = 0; d < 3; ++d) {
          double dv = 2.0 * (p.var[d] - f.velocity[d]);
          VShear[d] = VShear[d] + cinviscmult * dv;
        }
      }
    }
  }
  // AddBoundaryContributions_to_ME3D.f90:314-325
  if (c1_first) B_ren_inversion(p.Bg, o.prm.invb_det_thresh);
  if (Ncbf == 0) return;
  if (o.prm.c1_be) B_renormalise(p.Bg, gradpt);
  for (int d = 0; d < 3; ++d) {
    tpres[d] = tpres[d] + ALEt[d] + gradpt[d];
    tdiss[d] = tdiss[d] - VMon[d];
    tvisc[d] = tvisc[d] + VShear[d];
  }
}

// AddBoundaryContributions_to_ME2D.f90:96-402 (fixe/tapi, mode 1, C1/ALE3 off)
void AddBoundaryContributions_to_ME2D(Oracle& o, int npi, int IntNcbs, double* tpres, double* tdiss, double* tvisc) {
  const double pibmink = 10.0;
  Particle& p = o.pg[npi];
  const bool c1_first = o.prm.c1_be && o.on_going_time_step == 1;
  const int acix[2] = {0, 2};
  double ro0 = o.prm.den0, roi = p.dens, pressi = p.pres;
  double distpimin = o.prm.dx;
  double VMon[2] = {0, 0}, VShear[2] = {0, 0}, RG_sum[2] = {0, 0}, ALEt[3] = {0, 0, 0};
  int ibdt = o.BDP[3 * (npi - 1) + 2];
  for (int icbs = 1; icbs <= IntNcbs; ++icbs) {
    const BDT& e = o.BDTab[ibdt + icbs - 2];
    const Side& s = o.sides[e.CloBoNum - 1];
    const SphZone& z = o.zones[s.stretch - 1];
    double xpi = e.LocXYZ[0], ypi = e.LocXYZ[1];
    double IntWdS = e.BoundaryIntegral[0];
    double IntWdV = e.BoundaryIntegral[2];
    double IntWd1s0 = e.BoundaryIntegral[5];
    double IntWd3s0 = e.BoundaryIntegral[6];
    double GravN = 0.0, nnlocal[2], gradbPsuro[2];
    for (int i = 0; i < 2; ++i) {
      nnlocal[i] = s.T[acix[i]][2];
      gradbPsuro[i] = o.geff[acix[i]];
      GravN = GravN + o.geff[acix[i]] * nnlocal[i];
    }
    double sidevel[2];
    for (int i = 0; i < 2; ++i) sidevel[i] = (z.type == SPH_ZONE_TAPI) ? s.velocity[acix[i]] : 0.0;
    double Dvel[2];
    for (int i = 0; i < 2; ++i) Dvel[i] = 2.0 * (p.var[acix[i]] - sidevel[i]);
    double DvelN = Dvel[0] * nnlocal[0] + Dvel[1] * nnlocal[1];
    double distpi = std::max(ypi, distpimin);
    double pressib = pressi;
    double pressibmin = pibmink * ro0 * distpimin;
    if (DvelN <= 0.0) { if (pressib < pressibmin) pressib = pressibmin; }
    double PressB = pressib - ro0 * GravN * distpi;
    double QiiIntWdS = IntWdS * (pressib + PressB) / roi;
    double RG[2] = {0, 0};
    for (int i = 0; i < 2; ++i) {
      for (int j = 0; j < 2; ++j) RG[i] = RG[i] + s.RN[acix[i]][acix[j]] * gradbPsuro[j];
      RG[i] = RG[i] * IntWdV;
    }
    RG_sum[0] = RG_sum[0] + RG[0];
    RG_sum[1] = RG_sum[1] + RG[1];
    if (c1_first) {   // AddBoundaryContributions_to_ME2D.f90:290-300: -RN IntWdV
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) p.Bg[a][c] = p.Bg[a][c] + -s.RN[a][c] * IntWdV;
    }
    ALEt[0] = ALEt[0] - nnlocal[0] * QiiIntWdS;
    ALEt[2] = ALEt[2] - nnlocal[1] * QiiIntWdS;
    if (xpi >= 0.0 && xpi <= s.length) {
      double slip_coefficient = z.bc_shear_stress_input;
      double cinvisci = p.kin_visc;
      double Monvisc = o.prm.alfa_mon * o.celerita * o.h;
      double viscN = Monvisc;
      double TN = viscN * DvelN * IntWd3s0;
      double TT[2] = {TN * nnlocal[0], TN * nnlocal[1]};
      double SVforce;
      if (p.laminar_flag == 1 || !z.laminar_no_slip_check) SVforce = 2.0 * cinvisci * slip_coefficient * IntWd1s0;
      else SVforce = 0.0;
      double Dvel_Mor[3] = {2.0 * p.var[0], 2.0 * p.var[1], 2.0 * p.var[2]};
      for (int i = 0; i < 2; ++i) {
        VMon[i] = VMon[i] + TT[i];
        VShear[i] = VShear[i] + Dvel_Mor[acix[i]] * SVforce;
      }
    }
  }
  if (c1_first) B_ren_inversion(p.Bg, o.prm.invb_det_thresh);   // :377-383
  if (IntNcbs == 0) return;
  if (o.prm.c1_be) {   // :384-392: RG_sum renormalised with B_ren_gradp
    double aux2[3] = {RG_sum[0], 0.0, RG_sum[1]}, aux[3];
    for (int a = 0; a < 3; ++a) {
      double sum = 0.0;
      for (int c = 0; c < 3; ++c) sum = sum + p.Bg[a][c] * aux2[c];
      aux[a] = sum;
    }
    RG_sum[0] = -aux[0];
    RG_sum[1] = -aux[2];
  }
  for (int i = 0; i < 2; ++i) {
    tpres[acix[i]] = tpres[acix[i]] - RG_sum[i] - ALEt[acix[i]];
    tdiss[acix[i]] = tdiss[acix[i]] - VMon[i];
    tvisc[acix[i]] = tvisc[acix[i]] - VShear[i];
  }
}

// inter_EqMoto.f90:108-283 with viscomon.f90:54-73 and viscomorris.f90:60-71
// (Domain%tipo = "semi", liquid, time_stage = 1, all neighbours std)
void inter_EqMoto(Oracle& o, int npi, double* tpres, double* tdiss, double* tvisc) {
  Particle& p = o.pg[npi];
  const int NM = o.NMAXPARTJ;
  double rvw_sum[3] = {0, 0, 0}, t_pres_aux[3] = {0, 0, 0}, ALE1[3] = {0, 0, 0};
  for (int contj = 1; contj <= o.nPartIntorno[npi]; ++contj) {
    long npartint = (long)(npi - 1) * NM + contj;
    int npj = o.PartIntorno[npartint];
    if (npi == npj) continue;
    const Particle& q = o.pg[npj];
    double rhoi = p.dens, rhoj = q.dens, amassj = q.mass, pi = p.pres, pj = q.pres;
    double dervel[3] = {q.vel[0] - p.vel[0], q.vel[1] - p.vel[1], q.vel[2] - p.vel[2]};
    const double* rg = &o.rag[npartint * 3];
    const double* pk = &o.PartKernel[npartint * 4];
    double alpha = (pj - pi) / (rhoi * rhoj);
    double appopres[3];
    for (int d = 0; d < 3; ++d) appopres[d] = -(amassj * alpha * rg[d] * pk[2]);
    double alpha2 = (pi * (rhoj / rhoi + 1.0) + pj * (rhoi / rhoj - 1.0)) / (rhoi * rhoj);
    for (int d = 0; d < 3; ++d) ALE1[d] = ALE1[d] - amassj * alpha2 * rg[d] * pk[2];
    for (int d = 0; d < 3; ++d) t_pres_aux[d] = t_pres_aux[d] + appopres[d];
    // viscomon
    double vrij = -(dervel[0] * rg[0]) - dervel[1] * rg[1] - dervel[2] * rg[2];
    double rhotilde = p.dens + q.dens;
    double celtilde = o.celerita + o.celerita;
    double TermMon = o.prm.alfa_mon * celtilde * o.h / rhotilde;
    for (int d = 0; d < 3; ++d) {
      double rvwalfa = amassj * TermMon * vrij * rg[d] * pk[1];
      tdiss[d] = tdiss[d] + (rvwalfa + 0.0);
    }
    // viscomorris
    if (p.kin_visc > 1.0e-12 && q.kin_visc > 1.0e-12) {
      double rt = p.kin_visc * p.dens + q.kin_visc * q.dens + 1.0e-3;
      double anuitilde = 4.0 * (p.kin_visc * q.kin_visc);
      double factivis = amassj * anuitilde / rt;
      double rr = 0.0;
      for (int d = 0; d < 3; ++d) rr = rr + rg[d] * rg[d];
      for (int d = 0; d < 3; ++d) {
        double rvw = factivis * (-(dervel[d] * pk[1] * rr));
        tvisc[d] = tvisc[d] + rvw;
        rvw_sum[d] = rvw_sum[d] + rvw;
      }
    }
  }
  if (o.prm.c1_be) B_renormalise(p.Bg, t_pres_aux);   // inter_EqMoto.f90:255-260
  for (int d = 0; d < 3; ++d) tpres[d] = tpres[d] + t_pres_aux[d] + ALE1[d];
  p.laminar_flag = 0;
  if (p.kin_visc > 0.0) {
    double absv_pres = std::sqrt(tpres[0] * tpres[0] + tpres[1] * tpres[1] + tpres[2] * tpres[2]) + GI;
    double absv_Morris = std::sqrt(rvw_sum[0] * rvw_sum[0] + rvw_sum[1] * rvw_sum[1] + rvw_sum[2] * rvw_sum[2]);
    double weight = 0.0;
    if (absv_pres != 0.0) weight = absv_Morris / absv_pres * 100.0;
    p.laminar_flag = (weight > 5.0 || absv_pres == 0.0) ? 1 : 0;
  }
}

// AddElasticBoundaryReaction_3D.f90:67-154 (no convex edges)
// FindBoundaryConvexEdges3D.f90:64-150.  The reference runs the kf loop in
// parallel with the additions in a critical section, so its edge order
// depends on the threads; this is the order of a serial run.  After its
// first find for face nf the reference leaves the kf1 loop too (the second
// `if (EdgeFound) exit`), so every face contributes at most one edge.
void FindBoundaryConvexEdges3D(Oracle& o) {
  const int iseg[2][4] = {{2, 3, 1, 0}, {2, 3, 4, 1}};
  const int NumFacce = (int)o.BFaceList.size();
  o.BoundaryConvexEdge.clear();
  for (int kf = 1; kf <= NumFacce - 1; ++kf) {
    const int nf = o.BFaceList[kf - 1];
    const Face& F = o.faces[nf - 1];
    const int nodes = F.nodes, fk = nodes - 2;
    for (int kf1 = kf + 1; kf1 <= NumFacce; ++kf1) {
      const int nf1 = o.BFaceList[kf1 - 1];
      const Face& F1 = o.faces[nf1 - 1];
      const int nodes1 = F1.nodes, fk1 = nodes1 - 2;
      bool EdgeFound = false;
      for (int i = 1; i <= nodes; ++i) {
        const int j = iseg[fk - 1][i - 1];
        const int nodi = F.name[i - 1], nodj = F.name[j - 1];
        for (int ii = 1; ii <= nodes1; ++ii) {
          const int jj = iseg[fk1 - 1][ii - 1];
          const int nodii = F1.name[ii - 1], nodjj = F1.name[jj - 1];
          if ((nodi == nodii && nodj == nodjj) || (nodi == nodjj && nodj == nodii)) {
            const int kk = iseg[fk1 - 1][jj - 1];
            const int nodkk = F1.name[kk - 1];
            double zitakk = 0.0;
            for (int sd = 0; sd < 3; ++sd)
              zitakk = zitakk + F.T[sd][2] * (o.vert[3 * (nodkk - 1) + sd] - F.GX[nodes - 1][sd]);
            if (zitakk < 0.0) {
              ConvexEdge E;
              E.face[0] = nf;
              E.face[1] = nf1;
              double length2 = 0.0;
              for (int sd = 0; sd < 3; ++sd) {
                E.GX1[sd] = o.vert[3 * (nodi - 1) + sd];
                const double delta = o.vert[3 * (nodj - 1) + sd] - o.vert[3 * (nodi - 1) + sd];
                E.component[sd] = delta;
                length2 = length2 + delta * delta;
              }
              E.length = std::sqrt(length2);
              o.BoundaryConvexEdge.push_back(E);
              EdgeFound = true;
              break;
            }
          }
        }
        if (EdgeFound) break;
      }
      if (EdgeFound) break;
    }
  }
}

void AddElasticBoundaryReaction_3D(const Oracle& o, int npi, int Ncbf, double* R) {
  const Particle& p = o.pg[npi];
  R[0] = R[1] = R[2] = 0.0;
  double zimin = 0.25 * o.prm.dx;
  double celer02 = o.prm.eps / o.prm.den0;
  int ibdt = o.BDP[3 * (npi - 1) + 2];
  char rea_local[256];
  std::vector<char> rea_heap;
  char* ReaFace = rea_local;
  if (Ncbf > 256) {
    rea_heap.assign(Ncbf, 0);
    ReaFace = rea_heap.data();
  }
  for (int icbf = 1; icbf <= Ncbf; ++icbf) ReaFace[icbf - 1] = 0;
  for (int icbf = 1; icbf <= Ncbf; ++icbf) {
    const BDT& e = o.BDTab[ibdt + icbf - 2];
    const Face& f = o.faces[e.CloBoNum - 1];
    double zi = e.LocXYZ[2];
    if (zi < zimin) {
      double csi[3];
      LocalNormalCoordinates(f, e.LocXYZ, csi);
      if (IsPointInternal(f.nodes - 2, csi)) {
        double vin = 0.0;
        for (int sd = 0; sd < 3; ++sd) vin = vin + p.var[sd] * f.T[sd][2];
        if (vin < 0.0) {
          double normreact = -(1.0 * celer02 * std::log((o.h + zi - zimin) / o.h) / o.h);
          for (int d = 0; d < 3; ++d) R[d] = R[d] + normreact * f.T[d][2];
        }
        ReaFace[icbf - 1] = true;
      }
    }
  }
  // AddElasticBoundaryReaction_3D.f90:106-153: reaction from close convex edges
  for (const ConvexEdge& E : o.BoundaryConvexEdge) {
    int NCloseEdgeF = 0;
    for (int icbf = 1; icbf <= Ncbf; ++icbf) {
      const int iface = o.BDTab[ibdt + icbf - 2].CloBoNum;
      if (iface == E.face[0] && !ReaFace[icbf - 1]) NCloseEdgeF = NCloseEdgeF + 1;
      else if (iface == E.face[1] && !ReaFace[icbf - 1]) NCloseEdgeF = NCloseEdgeF + 1;
    }
    if (NCloseEdgeF != 2) return;
    double scaprod = 0.0;
    for (int sd = 0; sd < 3; ++sd) scaprod = scaprod + (p.coord[sd] - E.GX1[sd]) * E.component[sd];
    double edgelen2 = E.length * E.length;
    double tau = scaprod / edgelen2;
    if (tau >= 0.0 && tau <= 1.0) {
      double edgedist2 = 0.0, XQ[3], QP[3];
      for (int sd = 0; sd < 3; ++sd) XQ[sd] = E.GX1[sd] + E.component[sd] * tau;
      for (int sd = 0; sd < 3; ++sd) QP[sd] = p.coord[sd] - XQ[sd];
      for (int sd = 0; sd < 3; ++sd) edgedist2 = edgedist2 + QP[sd] * QP[sd];
      double zi = std::sqrt(edgedist2);
      if (zi < zimin) {
        double vin = 0.0, QPcosdir[3];
        for (int sd = 0; sd < 3; ++sd) QPcosdir[sd] = QP[sd] / zi;
        for (int sd = 0; sd < 3; ++sd) vin = vin + p.var[sd] * QPcosdir[sd];
        if (vin < 0.0) {
          double normreact = -(1.0 * celer02 * std::log(zi / zimin) / zimin);
          for (int sd = 0; sd < 3; ++sd) R[sd] = R[sd] + normreact * QPcosdir[sd];
        }
      }
    }
  }
}

// AddElasticBoundaryReaction_2D.f90:63-97
void AddElasticBoundaryReaction_2D(const Oracle& o, int npi, int Ncbs, double* R) {
  const Particle& p = o.pg[npi];
  R[0] = R[1] = R[2] = 0.0;
  double ypimin = 0.25 * o.prm.dx;
  double celer02 = o.prm.eps / o.prm.den0;
  int ibdt = o.BDP[3 * (npi - 1) + 2];
  for (int icbs = 1; icbs <= Ncbs; ++icbs) {
    const BDT& e = o.BDTab[ibdt + icbs - 2];
    const Side& s = o.sides[e.CloBoNum - 1];
    double xpi = e.LocXYZ[0], ypi = e.LocXYZ[1];
    if (ypi < ypimin && xpi > 0.0 && xpi < s.length) {
      double vin = 0.0;
      for (int sd = 0; sd < 3; ++sd) vin = vin + p.var[sd] * s.T[sd][2];
      if (vin < 0.0) {
        double normreact = -(1.0 * celer02 * std::log((o.h + ypi - ypimin) / o.h) / o.h);
        for (int sd = 0; sd < 3; ++sd) R[sd] = R[sd] + normreact * s.T[sd][2];
      }
    }
  }
}

// RHS_momentum_equation.f90:87-179
void RHS_momentum_equation(Oracle& o) {
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    double tpres[3] = {0, 0, 0}, tdiss[3] = {0, 0, 0}, tvisc[3] = {0, 0, 0};
    p.kodvel = 0;
    p.velass[0] = p.velass[1] = p.velass[2] = 0.0;
    int ncb = o.BDP[3 * (npi - 1)];
    int intn = o.BDP[3 * (npi - 1) + 1];
    bool active = (o.dim == 3) ? (ncb > 0) : (ncb > 0 && intn > 0);
    if (active || o.prm.c1_be) {   // RHS_momentum_equation.f90:133-150
      if (o.dim == 3) AddBoundaryContributions_to_ME3D(o, npi, ncb, tpres, tdiss, tvisc);
      else AddBoundaryContributions_to_ME2D(o, npi, intn, tpres, tdiss, tvisc);
    }
    inter_EqMoto(o, npi, tpres, tdiss, tvisc);
    if (active) {
      double R[3];
      if (o.dim == 3) AddElasticBoundaryReaction_3D(o, npi, ncb, R);
      else AddElasticBoundaryReaction_2D(o, npi, intn, R);
      for (int d = 0; d < 3; ++d) p.acc[d] = tpres[d] + tdiss[d] + tvisc[d] + o.geff[d] + R[d];
    } else {
      for (int d = 0; d < 3; ++d) p.acc[d] = tpres[d] + tdiss[d] + tvisc[d] + o.geff[d];
    }
  }
}

// ------------------------------------------------------------------------
// Time integration and EoS
// ------------------------------------------------------------------------

// time_step_duration.f90:59-123 (one liquid medium)
void time_step_duration(Oracle& o) {
  double dtmin = max_positive_number, dt_Mon = max_positive_number, dt_vis = max_positive_number;
  if (o.nag == 0) {
    o.dt = 0.0;
  } else {
    if (o.prm.kin_visc > 1.0e-24) {
      dt_vis = o.prm.vsc_coeff * o.squareh / (0.5 * o.prm.kin_visc);
      dtmin = std::min(dtmin, dt_vis);
    }
    double dmin = dtmin;
#pragma omp parallel for schedule(static) num_threads(o.nthreads) reduction(min:dmin)
    for (int npi = 1; npi <= o.nag; ++npi) {
      const Particle& p = o.pg[npi];
      double U = std::sqrt(p.vel[0] * p.vel[0] + p.vel[1] * p.vel[1] + p.vel[2] * p.vel[2]);
      double dt_CFL = o.prm.cfl * 2.0 * o.h / (o.celerita + U);
      dmin = std::min(dmin, std::min(dt_CFL, dt_vis));
    }
    dtmin = dmin;
    if (o.prm.dt_alfa_mon) {
      double visc_Mon = o.prm.alfa_mon * o.celerita * o.h / o.prm.den0;
      double dt_Mon_j = o.squareh / (0.5 * visc_Mon);
      dt_Mon = std::min(dt_Mon, dt_Mon_j);
      dtmin = std::min(dtmin, dt_Mon);
    }
    if (o.on_going_time_step == 0) o.dt = dtmin;
    else o.dt = (1.0 - o.prm.pesodt) * dtmin + o.prm.pesodt * o.dt_average;
  }
  if (o.on_going_time_step == 0) o.dt_average = o.dt;
  else o.dt_average = (o.dt_average * (o.on_going_time_step - 1) + o.dt) / o.on_going_time_step;
}

// Leapfrog_momentum.f90:66-99 followed by velocity_smoothing_2.f90:87-101
// with TetaV = 0 (var = vel)
void Leapfrog_momentum(Oracle& o, double dt_previous_step) {
  o.dtvel = 0.5 * (o.dt + dt_previous_step);
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    for (int d = 0; d < 3; ++d) p.vel[d] = p.vel[d] + o.dtvel * p.acc[d];
    if (p.kodvel == 1) p.vel[2] = p.velass[2];
    else if (p.kodvel == 2) for (int d = 0; d < 3; ++d) p.vel[d] = p.velass[d];
    for (int d = 0; d < 3; ++d) p.var[d] = p.vel[d];
  }
}

// Leapfrog_trajectories.f90:52-66
void Leapfrog_trajectories(Oracle& o) {
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.cella <= 0) continue;
    for (int d = 0; d < 3; ++d) p.coord[d] = p.coord[d] + o.dt * p.vel[d];
  }
}

// Leapfrog_continuity.f90:54-68 and EoS_fluid_loop.f90:59-69
void Leapfrog_continuity(Oracle& o) {
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.cella <= 0) continue;
    p.dens = p.dens + o.dt * p.dden;
    if (o.prm.density_thresholds == 1) {
      if (p.dens < 0.9 * o.prm.den0) p.dens = 0.9 * o.prm.den0;
      if (p.dens > 1.1 * o.prm.den0) p.dens = 1.1 * o.prm.den0;
    }
  }
}

void EoS_fluid_loop(Oracle& o) {
  if (o.on_going_time_step <= 0) return;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.cella <= 0) continue;
    p.pres = o.prm.eps / o.prm.den0 * (p.dens - o.prm.den0) + o.prm.p_ref;
  }
}

// velocity_smoothing.f90:85-132 with velocity_smoothing_SA_SPH_3D.f90:61-125 /
// _2D.f90:66-117 (wall zones fixe/tapi, slip mode 1), then
// velocity_smoothing_2.f90:68-102 for TetaV > 1e-9 (time_step_loop.f90:249-259)
void velocity_smoothing(Oracle& o) {
  const int NM = o.NMAXPARTJ;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    for (int d = 0; d < 3; ++d) p.var[d] = 0.0;
    for (int contj = 1; contj <= o.nPartIntorno[npi]; ++contj) {
      long npartint = (long)(npi - 1) * NM + contj;
      const Particle& q = o.pg[o.PartIntorno[npartint]];
      double rhoj = q.dens, amassj = q.mass;
      double dervel[3];
      for (int d = 0; d < 3; ++d) dervel[d] = q.vel[d] - p.vel[d];
      double pesoj = amassj * o.PartKernel[npartint * 4 + 3] / rhoj;
      for (int d = 0; d < 3; ++d) p.var[d] = p.var[d] + dervel[d] * pesoj;
    }
    int ibdt = o.BDP[3 * (npi - 1) + 2];
    if (o.dim == 3) {
      int Ncbf = o.BDP[3 * (npi - 1)];
      for (int icbf = 1; icbf <= Ncbf; ++icbf) {
        const BDT& e = o.BDTab[ibdt + icbf - 2];
        const Face& f = o.faces[e.CloBoNum - 1];
        const SphZone& z = o.zones[f.stretch - 1];
        double DVGlo[3], DVLoc[3], BCLoc[3];
        for (int i = 0; i < 3; ++i) DVGlo[i] = 2.0 * (f.velocity[i] - p.vel[i]);   // Tratto%velocity (0 for fixe)
        for (int i = 0; i < 3; ++i) {
          DVLoc[i] = 0.0;
          for (int j = 0; j < 3; ++j) DVLoc[i] = DVLoc[i] + f.T[j][i] * DVGlo[j];
        }
        double IntWdV = e.BoundaryIntegral[1];
        double slip = z.bc_shear_stress_input;
        BCLoc[0] = DVLoc[0] * IntWdV * slip;
        BCLoc[1] = DVLoc[1] * IntWdV * slip;
        BCLoc[2] = DVLoc[2] * IntWdV;
        for (int i = 0; i < 3; ++i) {
          double g = 0.0;
          for (int j = 0; j < 3; ++j) g = g + f.T[i][j] * BCLoc[j];
          p.var[i] = p.var[i] + g;
        }
      }
    } else {
      int IntNcbs = o.BDP[3 * (npi - 1) + 1];
      const int acix[2] = {0, 2};
      for (int icbs = 1; icbs <= IntNcbs; ++icbs) {
        const BDT& e = o.BDTab[ibdt + icbs - 2];
        const Side& sd = o.sides[e.CloBoNum - 1];
        const SphZone& z = o.zones[sd.stretch - 1];
        double sss[2], nnn[2], DVGlo[2], DVLoc[2], BCLoc[2], BCGlo[2];
        for (int i = 0; i < 2; ++i) {
          sss[i] = sd.T[acix[i]][0];
          nnn[i] = sd.T[acix[i]][2];
          DVGlo[i] = 2.0 * (sd.velocity[acix[i]] - p.vel[acix[i]]);   // Tratto%velocity (0 for fixe)
        }
        DVLoc[0] = sss[0] * DVGlo[0] + sss[1] * DVGlo[1];
        DVLoc[1] = nnn[0] * DVGlo[0] + nnn[1] * DVGlo[1];
        double IntWdV = e.BoundaryIntegral[2];
        double slip = z.bc_shear_stress_input;
        BCLoc[0] = DVLoc[0] * IntWdV * slip;
        BCLoc[1] = DVLoc[1] * IntWdV;
        BCGlo[0] = sss[0] * BCLoc[0] + nnn[0] * BCLoc[1];
        BCGlo[1] = sss[1] * BCLoc[0] + nnn[1] * BCLoc[1];
        p.var[0] = p.var[0] + BCGlo[0];
        p.var[2] = p.var[2] + BCGlo[1];
      }
    }
  }
  const double TetaV1 = o.prm.teta_v * o.celerita * o.dt / o.h;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.kodvel == 0) {
      for (int d = 0; d < 3; ++d) p.var[d] = p.vel[d] + TetaV1 * p.var[d];
      for (int d = 0; d < 3; ++d) p.vel[d] = p.var[d];
    } else {
      for (int d = 0; d < 3; ++d) p.var[d] = p.vel[d];
    }
  }
}

// PressureSmoothing_3D.f90:88-160 / PressureSmoothing_2D.f90:102-235
// (SmoothVersion "b"; wall zones fixe/tapi), time_step_loop.f90:397-404
void PressureSmoothing(Oracle& o) {
  const int NM = o.NMAXPARTJ;
  std::vector<double> vpres(o.nag + 1, 0.0);
  const double TetaP1 = o.prm.teta_p * o.celerita * o.dt / o.h;
  const double p0i = o.prm.p_ref, ro0i = o.prm.den0;
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.koddens != 0) continue;
    int Nsp = o.nPartIntorno[npi];
    double pi = p.pres, sompW = 0.0, AppUnity = 0.0;
    for (int j = 1; j <= Nsp; ++j) {
      long npartint = (long)(npi - 1) * NM + j;
      const Particle& q = o.pg[o.PartIntorno[npartint]];
      double pesoj = q.mass * o.PartKernel[npartint * 4 + 3] / q.dens;
      AppUnity = AppUnity + pesoj;
      sompW = sompW + (q.pres - pi) * pesoj;
    }
    int ibdt = o.BDP[3 * (npi - 1) + 2];
    if (o.dim == 3) {
      double DiffP = 0.0;
      if (Nsp > 0) {
        int Ncbf = o.BDP[3 * (npi - 1)];
        for (int icbf = 1; icbf <= Ncbf; ++icbf) {
          const BDT& e = o.BDTab[ibdt + icbf - 2];
          if (e.LocXYZ[2] > 0.0) AppUnity = AppUnity + e.BoundaryIntegral[1];
        }
        if (AppUnity < 0.95) DiffP = sompW + (p0i - pi) * (1.0 - AppUnity);
        else DiffP = sompW / AppUnity;
      }
      vpres[npi] = pi + TetaP1 * DiffP;
    } else {
      if (Nsp <= 0) {
        vpres[npi] = pi;
        continue;
      }
      const int acix[2] = {0, 2};
      double VIntWdV_FT = 0.0;
      int IntNcbs = o.BDP[3 * (npi - 1) + 1];
      for (int icbs = 1; icbs <= IntNcbs; ++icbs) {
        const BDT& e = o.BDTab[ibdt + icbs - 2];
        const Side& sd = o.sides[e.CloBoNum - 1];
        double sss[2], nnn[2], mf[2];
        for (int i = 0; i < 2; ++i) {
          sss[i] = sd.T[acix[i]][0];
          nnn[i] = sd.T[acix[i]][2];
        }
        mf[0] = sss[0] * o.geff[acix[0]] + sss[1] * o.geff[acix[1]];
        mf[1] = nnn[0] * o.geff[acix[0]] + nnn[1] * o.geff[acix[1]];
        VIntWdV_FT = VIntWdV_FT + e.BoundaryIntegral[1];
        sompW = sompW + ro0i * (mf[0] * e.BoundaryIntegral[3] + mf[1] * e.BoundaryIntegral[4]);
      }
      AppUnity = AppUnity + VIntWdV_FT + 0.0 + 0.0 + 0.0;
      vpres[npi] = pi + TetaP1 * (sompW + (pi - pi) * 0.0 + (pi - pi) * 0.0 + (p0i - pi) * (1.0 - AppUnity));
    }
  }
#pragma omp parallel for schedule(static) num_threads(o.nthreads)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    if (p.koddens != 0) continue;
    p.pres = vpres[npi];
    p.dens = o.prm.den0 * (1.0 + (p.pres - o.prm.p_ref) / o.prm.eps);   // EoS_barotropic_linear.f90:54
  }
}

// time_step_loop.f90:338-360
int continuity_block(Oracle& o) {
  int ncbfmax = 0;
#pragma omp parallel for schedule(static) num_threads(o.nthreads) reduction(max:ncbfmax)
  for (int npi = 1; npi <= o.nag; ++npi) {
    Particle& p = o.pg[npi];
    p.dden = 0.0;
    p.koddens = 0;
    int loc = 0;
    SASPH_continuity(o, npi, loc);
    ncbfmax = std::max(ncbfmax, loc);
    Continuity_Equation(o, npi);
  }
  o.Ncbf_Max = ncbfmax;
  if (o.dim == 3 && ncbfmax > o.maxcb) return SPH_ERR_NCBF_MAX;
  return 0;
}

int boundary_tab(Oracle& o) {
  return (o.dim == 3) ? ComputeBoundaryDataTab_3D(o) : ComputeBoundaryDataTab_2D(o);
}

int check(Oracle& o, int st) { if (st && !o.fatal) o.fatal = st; return st; }

}  // namespace

// ------------------------------------------------------------------------
// C interface (test infrastructure)
// ------------------------------------------------------------------------
extern "C" {

void* ora_create(const SphParams* prm, const SphGeometry* g, int n, const double* x, const double* v,
                 const double* rho, const double* p, const double* m, int nthreads) {
  Oracle* o = new Oracle();
  o->prm = *prm;
  set_body_force(*o, 0.0);
  o->dim = prm->dim;
  o->ncord = prm->dim;
  o->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  // ReadInput.f90:198-205
  o->h = prm->dx * prm->trunc;
  o->doubleh = 2.0 * o->h;
  o->squareh = o->h * o->h;
  o->square_doubleh = o->doubleh * o->doubleh;
  o->unosuh = 1.0 / o->h;
  o->unosusquareh = 1.0 / o->squareh;
  o->eta = 1.0e-3 * o->h;
  o->eta2 = 1.0e-2 * o->squareh;
  // Gest_Input.f90:266-289
  double hp = (o->dim == 3) ? sq3(o->h) : o->h * o->h;
  o->coefke = ((o->dim == 3) ? 0.477464 : 0.682093) / hp;
  o->coefkacl = ((o->dim == 3) ? 0.074603 : 0.099472) / hp;
  double r = o->h * 4.0 / prm->dx;
  double rp = (o->dim == 3) ? sq3(r) : r * r;
  o->NMAXPARTJ = (int)(prm->coef_nmaxpartj * rp) + 1;
  o->celerita = std::sqrt(prm->eps / prm->den0);   // ReadInputMedium.f90:156
  o->maxcb = (o->dim == 3) ? prm->max_close_bound_faces : MAXCLOSEBOUNDSIDES;
  CreaGrid(*o);
  // geometry
  o->zones.assign(g->zones, g->zones + g->n_zones);
  o->vert.assign(g->vertices, g->vertices + 3 * g->n_vertices);
  if (o->dim == 3) {
    o->faces.resize(g->n_faces);
    for (int f = 0; f < g->n_faces; ++f) {
      Face& F = o->faces[f];
      std::memset(&F, 0, sizeof(Face));
      int nn = 0;
      for (int k = 0; k < 4; ++k) { F.name[k] = g->face_nodes[4 * f + k]; if (F.name[k] > 0) nn++; }
      F.nodes = nn;
      F.stretch = g->face_zone[f];
      DefineLocalSystemVersors(*o, F);
      const SphZone& z = o->zones[F.stretch - 1];
      for (int d = 0; d < 3; ++d) F.velocity[d] = (z.type == SPH_ZONE_TAPI) ? z.velocity[d] : 0.0;
    }
    // CompleteBoundaries3D.f90: faces ordered by zone
    for (int nt = 1; nt <= g->n_zones; ++nt)
      for (int f = 0; f < g->n_faces; ++f)
        if (o->faces[f].stretch == nt) o->BFaceList.push_back(f + 1);
    FindBoundaryConvexEdges3D(*o);
    GridCellBoundaryFacesIntersections3D(*o);
    ComputeBoundaryIntegralTab(*o);
    ComputeKernelTable(*o);
  } else {
    o->sides.resize(g->n_sides);
    for (int s = 0; s < g->n_sides; ++s) {
      o->sides[s].vertex[0] = g->side_vertices[2 * s];
      o->sides[s].vertex[1] = g->side_vertices[2 * s + 1];
      o->sides[s].stretch = g->side_zone[s];
    }
    DefineBoundarySideGeometry2D(*o);
    for (int i = 0; i < 22; ++i) for (int j = 0; j < 6; ++j) o->BIT2D[i][j] = (double)BIT2D_LIT[i][j];
  }
  // particles
  o->nag = n;
  o->pg.assign(n + 2, Particle{});
  for (int i = 0; i < n; ++i) {
    Particle& q = o->pg[i + 1];
    for (int d = 0; d < 3; ++d) { q.coord[d] = x[3 * i + d]; q.vel[d] = v[3 * i + d]; q.var[d] = v[3 * i + d]; }
    q.dens = rho[i]; q.pres = p[i]; q.mass = m[i];
    q.kin_visc = prm->kin_visc;
  }
  o->Icont.assign(o->nmax + 2, 0);
  o->NPartOrd.assign(n + 2, 0);
  o->nPartIntorno.assign(n + 2, 0);
  long slots = (long)o->NMAXPARTJ * n + 1;
  o->PartIntorno.assign(slots, 0);
  o->PartKernel.assign(slots * 4, 0.0);
  o->rag.assign(slots * 3, 0.0);
  o->BDP.assign(3 * (size_t)n + 3, 0);
  o->BDTab.assign((size_t)o->maxcb * n + 1, BDT{});
  return o;
}

void ora_destroy(void* h) { delete static_cast<Oracle*>(h); }

int ora_nmaxpartj(void* h) { return static_cast<Oracle*>(h)->NMAXPARTJ; }
int ora_n(void* h) { return static_cast<Oracle*>(h)->nag; }
int ora_nmax(void* h) { return static_cast<Oracle*>(h)->nmax; }
int ora_truncated(void* h) { return static_cast<Oracle*>(h)->truncated; }
int ora_removed(void* h) { return static_cast<Oracle*>(h)->EpOrdGrid; }
int ora_ncbf_max(void* h) { return static_cast<Oracle*>(h)->Ncbf_Max; }
double ora_dt(void* h) { return static_cast<Oracle*>(h)->dt; }
double ora_forcing_sin(double x) { return forcing_sin(x); }
double ora_time(void* h) { return static_cast<Oracle*>(h)->simulation_time; }
int ora_step_index(void* h) { return static_cast<Oracle*>(h)->on_going_time_step; }
void ora_grid_info(void* h, int* ncd, double* extr_lo, double* dcd) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int d = 0; d < 3; ++d) { ncd[d] = o->ncd[d]; extr_lo[d] = o->extr[d][0]; dcd[d] = o->dcd[d]; }
}

// IC part of time_step_loop.f90:82-173 (OrdGrid1 from Gest_Input.f90:591)
int ora_prepare(void* h) {
  Oracle& o = *static_cast<Oracle*>(h);
  OrdGrid1(o);
  CalcVarLength(o);
  int st = boundary_tab(o);
  if (st) return check(o, st);
  o.on_going_time_step = -999;
  time_step_duration(o);
  set_body_force(o, o.simulation_time + o.dt);
  return 0;
}

// Neighbour search + boundary data at the current positions (no IC dt).
int ora_search(void* h) {
  Oracle& o = *static_cast<Oracle*>(h);
  OrdGrid1(o);
  CalcVarLength(o);
  return check(o, boundary_tab(o));
}

// RHS_momentum_equation as time_step_loop.f90 calls it, after advancing
// on_going_time_step: a call between steps evaluates the momentum of the
// next step (which matters only for the step-1 completion of B_ren_gradp).
int ora_rhs_momentum(void* h) {
  Oracle& o = *static_cast<Oracle*>(h);
  const int saved = o.on_going_time_step;
  o.on_going_time_step = saved < 0 ? 1 : saved + 1;
  RHS_momentum_equation(o);
  o.on_going_time_step = saved;
  return 0;
}
int ora_continuity(void* h) { Oracle& o = *static_cast<Oracle*>(h); return check(o, continuity_block(o)); }
int ora_time_step_duration(void* h) { time_step_duration(*static_cast<Oracle*>(h)); return 0; }

// time_step_loop.f90:175-405, leapfrog, one step per iteration
int ora_step(void* h, int nsteps) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int s = 0; s < nsteps; ++s) {
    int it = (o.on_going_time_step < 0) ? 1 : o.on_going_time_step + 1;
    o.on_going_time_step = it;
    double dt_previous_step = o.dt;
    time_step_duration(o);
    o.simulation_time = o.simulation_time + o.dt;
    set_body_force(o, o.simulation_time);
    RHS_momentum_equation(o);
    Leapfrog_momentum(o, dt_previous_step);
    if (o.prm.teta_v > 1.0e-9) velocity_smoothing(o);
    Leapfrog_trajectories(o);
    OrdGrid1(o);
    CalcVarLength(o);
    int st = boundary_tab(o);
    if (st) return check(o, st);
    st = continuity_block(o);
    if (st) return check(o, st);
    Leapfrog_continuity(o);
    EoS_fluid_loop(o);
    if (o.prm.teta_p > 0.0) PressureSmoothing(o);
  }
  return 0;
}

// State in pg order.  Any pointer may be NULL.
int ora_get(void* h, double* x, double* v, double* rho, double* p, double* m, double* acc, double* dden) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 0; i < o.nag; ++i) {
    const Particle& q = o.pg[i + 1];
    for (int d = 0; d < 3; ++d) {
      if (x) x[3 * i + d] = q.coord[d];
      if (v) v[3 * i + d] = q.vel[d];
      if (acc) acc[3 * i + d] = q.acc[d];
    }
    if (rho) rho[i] = q.dens;
    if (p) p[i] = q.pres;
    if (m) m[i] = q.mass;
    if (dden) dden[i] = q.dden;
  }
  return o.nag;
}

// fluid_global_quantities.f90:59-72: mass, linear momentum, angular momentum
// about the origin (Vector_Product of coord and vel) and volume sum(m / rho)
// over pg(1:nag), summed sequentially in pg order.  out[0] mass, out[1..3]
// linear momentum, out[4..6] angular momentum, out[7] volume.
void ora_global_quantities(void* h, double* out) {
  Oracle& o = *static_cast<Oracle*>(h);
  double glob_mass = 0.0, glob_vol = 0.0, lin[3] = {0, 0, 0}, ang[3] = {0, 0, 0}, aux[3];
  for (int ip = 1; ip <= o.nag; ++ip) {
    const Particle& q = o.pg[ip];
    glob_mass = glob_mass + q.mass;
    for (int d = 0; d < 3; ++d) lin[d] = lin[d] + q.mass * q.vel[d];
    Vector_Product(q.coord, q.vel, aux);
    for (int d = 0; d < 3; ++d) ang[d] = ang[d] + q.mass * aux[d];
    glob_vol = glob_vol + q.mass / q.dens;
  }
  out[0] = glob_mass;
  for (int d = 0; d < 3; ++d) { out[1 + d] = lin[d]; out[4 + d] = ang[d]; }
  out[7] = glob_vol;
}

// The renormalisation matrices B_ren_gradp and B_ren_divu in pg order, 9
// doubles per particle, B(i,j) at [9 k + 3 i + j].  Either pointer may be NULL.
int ora_get_c1(void* h, double* bg, double* bd) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 0; i < o.nag; ++i) {
    const Particle& q = o.pg[i + 1];
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        if (bg) bg[9 * i + 3 * a + c] = q.Bg[a][c];
        if (bd) bd[9 * i + 3 * a + c] = q.Bd[a][c];
      }
  }
  return o.nag;
}

// The convex edges FindBoundaryConvexEdges3D found: their count, and the
// two face ids of each in faces[2 * ne], [2 * ne + 1] (faces may be NULL).
int ora_convex_edges(void* h, int* faces) {
  Oracle& o = *static_cast<Oracle*>(h);
  const int ne = (int)o.BoundaryConvexEdge.size();
  if (faces)
    for (int e = 0; e < ne; ++e) {
      faces[2 * e] = o.BoundaryConvexEdge[e].face[0];
      faces[2 * e + 1] = o.BoundaryConvexEdge[e].face[1];
    }
  return ne;
}

int ora_laminar(void* h, int* flags) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 0; i < o.nag; ++i) flags[i] = o.pg[i + 1].laminar_flag;
  return o.nag;
}

int ora_grid(void* h, int* cella, int* icont, int* npartord) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 0; i < o.nag; ++i) {
    if (cella) cella[i] = o.pg[i + 1].cella;
    if (npartord) npartord[i] = o.NPartOrd[i + 1];
  }
  if (icont) for (int c = 1; c <= o.nmax + 1; ++c) icont[c - 1] = o.Icont[c];
  return 0;
}

int ora_neighbours(void* h, int nmaxj, int* counts, int* lists) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 1; i <= o.nag; ++i) {
    int c = o.nPartIntorno[i];
    counts[i - 1] = c;
    if (lists)
      for (int k = 0; k < c && k < nmaxj; ++k)
        lists[(long)(i - 1) * nmaxj + k] = o.PartIntorno[(long)(i - 1) * o.NMAXPARTJ + k + 1];
  }
  return 0;
}

// PartKernel(1:4) and rag(1:3) of slot k of particle i: out[(i*nmaxj+k)*7 + ...]
int ora_pair_data(void* h, int nmaxj, double* out) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 1; i <= o.nag; ++i)
    for (int k = 0; k < o.nPartIntorno[i] && k < nmaxj; ++k) {
      long s = (long)(i - 1) * o.NMAXPARTJ + k + 1;
      double* d = &out[((long)(i - 1) * nmaxj + k) * 7];
      for (int q = 0; q < 4; ++q) d[q] = o.PartKernel[s * 4 + q];
      for (int q = 0; q < 3; ++q) d[4 + q] = o.rag[s * 3 + q];
    }
  return 0;
}

int ora_boundary(void* h, int max_per, int* ncb, int* clobonum, double* values) {
  Oracle& o = *static_cast<Oracle*>(h);
  for (int i = 1; i <= o.nag; ++i) {
    int n = (o.dim == 3) ? o.BDP[3 * (i - 1)] : o.BDP[3 * (i - 1) + 1];
    ncb[i - 1] = n;
    int base = o.BDP[3 * (i - 1) + 2];
    for (int k = 0; k < n && k < max_per; ++k) {
      const BDT& e = o.BDTab[base + k - 1];
      clobonum[(long)(i - 1) * max_per + k] = e.CloBoNum;
      double* d = &values[((long)(i - 1) * max_per + k) * 20];
      for (int q = 0; q < 3; ++q) d[q] = e.LocXYZ[q];
      for (int q = 0; q < 8; ++q) d[3 + q] = e.BoundaryIntegral[q];
      for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) d[11 + 3 * c + r] = e.IntGiWrRdV[r][c];
    }
  }
  return 0;
}

// IC tables for known-answer tests.
void ora_tables(void* h, double* kerneltab /*41x5*/, double* bit /*256x7*/, double* bit2d /*22x6*/) {
  Oracle& o = *static_cast<Oracle*>(h);
  if (kerneltab) std::memcpy(kerneltab, o.kerneltab, sizeof(o.kerneltab));
  if (bit) std::memcpy(bit, o.BIT, sizeof(o.BIT));
  if (bit2d) for (int i = 0; i < 22; ++i) for (int j = 0; j < 6; ++j) bit2d[6 * i + j] = (double)BIT2D_LIT[i][j];
}

double ora_IWro2dro(double ro) { return IWro2dro(ro); }
double ora_JdWsRn(double ro, int n) { return JdWsRn(ro, n); }
double ora_WIntegr(double ri, double hh) { return WIntegr(ri, hh); }
double ora_J2Wro2(double ro) { return J2Wro2(ro); }
double ora_w(double r, double h, double coef) { return w_kernel(r, h, coef); }

}  // extern "C"
