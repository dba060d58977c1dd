// Allocation-free variant of the OrdGrid1 binning and counting sort.
//
// Why it exists: some callers cannot let a library call cudaMalloc --
// for example a Fortran host whose device arrays come from its own pool
// allocator (CUDA Fortran / OpenACC data regions) and which forbids
// allocations behind its back, or a time loop that must not hit the
// implicit device synchronisation cudaMalloc/cudaFree can cause.  This
// entry point takes device pointers for its inputs and outputs and keeps
// its working memory in a fixed, file-scope device array instead.
//
// Limits: at most kStaticMaxParticles particles and kStaticMaxCells grid
// cells per call.  The scratch array (about 20 MB) is part of the module:
// every GPU that loads the library holds it until the process exits.
//
// Sharing: every call uses the same array, so calls whose work overlaps on
// the GPU (concurrent streams, or host threads driving the same device)
// race on it and must be serialised by the caller.  The array keeps the
// contents of the previous call; the counters are cleared at the start of
// each call.
//
// Set-up: the first call in a device's context looks up the array's device
// address (cudaGetSymbolAddress, which may load the module) and must come
// before any stream capture on that device; later calls reuse the address
// until the context changes (a cudaDeviceReset), when it is looked up again.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/sphera_b200.h"

namespace {

constexpr int kStaticMaxParticles = 1 << 20;
constexpr int kStaticMaxCells = 1 << 20;
constexpr int kThreads = 256;
constexpr int kScanChunk = 4096;
constexpr int kMaxScanBlocks = (kStaticMaxCells + 1 + kScanChunk - 1) / kScanChunk;

// counts[kStaticMaxCells + 1] | starts[kStaticMaxCells + 1] |
// slot[kStaticMaxParticles] | tmp_id[kStaticMaxParticles] | scan[kMaxScanBlocks + 1]
constexpr size_t kScratchInts = 2 * ((size_t)kStaticMaxCells + 1) + 2 * (size_t)kStaticMaxParticles +
                                (size_t)kMaxScanBlocks + 1;

static __device__ __align__(256) int g_ordgrid_scratch[kScratchInts];

struct GridConst {
  double extr_lo[3];
  double dcd[3];
  int ncd[3];
  int dim;
  int ncells;
};

// ParticleCellNumber.f90:52-62 with CellNumber.f90:53-59 (1-based, 0 outside)
__device__ __forceinline__ int ref_cell(const GridConst& g, double x, double y, double z) {
  double ci = ceil((x - g.extr_lo[0]) / g.dcd[0]);
  double ck = ceil((z - g.extr_lo[2]) / g.dcd[2]);
  double cj = (g.dim == 3) ? ceil((y - g.extr_lo[1]) / g.dcd[1]) : 1.0;
  if (!(ci >= 1.0 && ci <= (double)g.ncd[0] && cj >= 1.0 && cj <= (double)g.ncd[1] && ck >= 1.0 &&
        ck <= (double)g.ncd[2]))
    return 0;
  return (((int)ck - 1) * g.ncd[1] + ((int)cj - 1)) * g.ncd[0] + (int)ci;
}

__global__ void k_static_clear(int* counts, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) counts[i] = 0;
}

__global__ void k_static_bin(GridConst g, int n, const double* __restrict__ x, int* cella, int* counts, int* slot) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = ref_cell(g, x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2]);
  cella[i] = c;
  slot[i] = (c > 0) ? atomicAdd(counts + c - 1, 1) : -1;
}

__device__ __forceinline__ int block_scan(int v, int* ws, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int s = lane < nw ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  int base = wid > 0 ? ws[wid - 1] : 0;
  total = ws[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

// Icont(1:nmax+1) of OrdGrid1.f90:87-94: 1-based exclusive starts.
__global__ void __launch_bounds__(1024) k_static_scan1(const int* counts, int n, int* bsum) {
  __shared__ int ws[32];
  int base = blockIdx.x * kScanChunk + threadIdx.x * 4;
  int v = 0;
  for (int q = 0; q < 4; ++q) v += (base + q < n) ? counts[base + q] : 0;
  int total;
  block_scan(v, ws, total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_static_scan2(int* bsum, int nb) {
  __shared__ int ws[32];
  int carry = 0;
  for (int c0 = 0; c0 < nb; c0 += 1024) {
    int i = c0 + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    int total;
    int ex = block_scan(v, ws, total);
    if (i < nb) bsum[i] = ex + carry;
    carry += total;
  }
}

__global__ void __launch_bounds__(1024) k_static_scan3(const int* counts, int n, const int* bsum, int* starts,
                                                       int* icont) {
  __shared__ int ws[32];
  int base = blockIdx.x * kScanChunk + threadIdx.x * 4;
  int vals[4];
  int v = 0;
  for (int q = 0; q < 4; ++q) {
    vals[q] = (base + q < n) ? counts[base + q] : 0;
    v += vals[q];
  }
  int total;
  int ex = block_scan(v, ws, total) + bsum[blockIdx.x];
  for (int q = 0; q < 4; ++q) {
    if (base + q < n) {
      starts[base + q] = ex;
      icont[base + q] = ex + 1;
    }
    ex += vals[q];
  }
}

// Unstable placement, then the rank of each particle index inside its cell
// (OrdGrid1.f90:100-105 scatters in increasing particle index).
__global__ void k_static_place(int n, const int* cella, const int* slot, const int* starts, int* tmp_id) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cella[i] <= 0) return;
  tmp_id[starts[cella[i] - 1] + slot[i]] = i + 1;
}

__global__ void k_static_rank(int n, const int* cella, const int* slot, const int* starts, const int* counts,
                              const int* tmp_id, int* npartord) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || cella[i] <= 0) return;
  int c = cella[i] - 1;
  int cs = starts[c], ce = cs + counts[c];
  int rank = 0;
  for (int q = cs; q < ce; ++q) rank += (tmp_id[q] < i + 1) ? 1 : 0;
  npartord[cs + rank] = i + 1;
}

__global__ void k_static_tail(int* icont, int ncells, const int* bsum, int nb, const int* counts) {
  // Icont(nmax+1) = number of particles in the grid + 1
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    (void)bsum;
    (void)nb;
    int last = icont[ncells - 1] - 1 + counts[ncells - 1];
    icont[ncells] = last + 1;
  }
}

// Scratch address of each device, taken once per device context
// (cudaGetSymbolAddress must run with that device current).  The entry is
// keyed on the context's process-unique id (cuCtxGetId, reached through
// cudaGetDriverEntryPoint so the library needs no libcuda link): after a
// cudaDeviceReset the runtime creates a new primary context, the module and
// its array are loaded again, possibly at another address, and the next
// call looks the address up afresh instead of using the old one.  A mutex
// makes the check-then-store safe when several host threads call at once.
constexpr int kMaxDevices = 64;
struct ScratchEntry {
  unsigned long long ctx_id;
  int* ptr;
};
ScratchEntry g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mutex;

typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

// Id of the context current on this thread; false if none can be had.
bool current_context_id(unsigned long long* id) {
  static PfnCtxGetCurrent get_current = nullptr;
  static PfnCtxGetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      cudaGetLastError();
      return false;
    }
    get_current = (PfnCtxGetCurrent)f1;
    get_id = (PfnCtxGetId)f2;
  }
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
  return get_id(ctx, id) == CUDA_SUCCESS;
}

// The device address of g_ordgrid_scratch in the current context of
// device dev (looked up on the first call in that context).
int scratch_address(int dev, int** out) {
  unsigned long long id = 0;
  if (!current_context_id(&id)) {
    // no context current on this thread yet: cudaSetDevice initialises the
    // device's primary context and makes it current, the context the
    // kernels of this call will run in
    if (cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      return SPH_ERR_NO_DEVICE;
    }
    if (!current_context_id(&id)) return SPH_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  ScratchEntry& e = g_scratch[dev];
  if (!e.ptr || e.ctx_id != id) {
    int* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_ordgrid_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return SPH_ERR_CUDA;
    }
    e.ptr = p;
    e.ctx_id = id;
  }
  *out = e.ptr;
  return SPH_OK;
}

}  // namespace

extern "C" int sph_ord_grid_static(const SphParams* params, int32_t n, const double* d_x, int32_t* d_cella,
                                   int32_t* d_icont, int32_t* d_npartord, void* stream) {
  if (!params || n < 0 || (n > 0 && (!d_x || !d_cella || !d_npartord)) || !d_icont) return SPH_ERR_INVALID_ARGUMENT;
  if (params->dim != 2 && params->dim != 3) return SPH_ERR_INVALID_ARGUMENT;
  if (!(params->dx > 0.0) || !(params->trunc > 0.0)) return SPH_ERR_INVALID_ARGUMENT;
  if (n > kStaticMaxParticles) return SPH_ERR_INVALID_ARGUMENT;
  // CreaGrid.f90:51-74
  GridConst g;
  std::memset(&g, 0, sizeof(g));
  g.dim = params->dim;
  double h = params->dx * params->trunc;
  double doubleh = 2.0 * h;
  double epsi = 0.01 * params->dx;
  for (int d = 0; d < 3; ++d) {
    double lo = params->domain_lo[d] - doubleh - epsi;
    double hi = params->domain_hi[d] + doubleh + epsi;
    double dextr = hi - lo;
    g.extr_lo[d] = lo;
    g.ncd[d] = (int)std::lround(dextr / doubleh);
    if (g.ncd[d] < 1) return SPH_ERR_INVALID_ARGUMENT;
    g.dcd[d] = dextr / g.ncd[d];
  }
  if (g.dim == 2) g.ncd[1] = 1;
  long long nc = (long long)g.ncd[0] * g.ncd[1] * g.ncd[2];
  if (nc > kStaticMaxCells) return SPH_ERR_INVALID_ARGUMENT;
  g.ncells = (int)nc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return SPH_ERR_NO_DEVICE;
  }
  // set-up on the first call in this device's context (that call must not
  // be inside a stream capture)
  int* base = nullptr;
  {
    int st = scratch_address(dev, &base);
    if (st != SPH_OK) return st;
  }
  int* counts = base;
  int* starts = counts + (kStaticMaxCells + 1);
  int* slot = starts + (kStaticMaxCells + 1);
  int* tmp_id = slot + kStaticMaxParticles;
  int* bsum = tmp_id + kStaticMaxParticles;
  cudaStream_t st = (cudaStream_t)stream;
  int ncells = g.ncells;
  int nb = (ncells + kScanChunk - 1) / kScanChunk;
  k_static_clear<<<256, kThreads, 0, st>>>(counts, ncells + 1);
  if (n > 0) k_static_bin<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(g, n, d_x, d_cella, counts, slot);
  k_static_scan1<<<nb, 1024, 0, st>>>(counts, ncells, bsum);
  k_static_scan2<<<1, 1024, 0, st>>>(bsum, nb);
  k_static_scan3<<<nb, 1024, 0, st>>>(counts, ncells, bsum, starts, d_icont);
  k_static_tail<<<1, 32, 0, st>>>(d_icont, ncells, bsum, nb, counts);
  if (n > 0) {
    k_static_place<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(n, d_cella, slot, starts, tmp_id);
    k_static_rank<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(n, d_cella, slot, starts, counts, tmp_id,
                                                                       d_npartord);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}
