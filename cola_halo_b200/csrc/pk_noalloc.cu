// Power-spectrum shell sums that allocate nothing.
//
// Some callers cannot allocate device memory at the point where they want a
// power spectrum: code running inside a memory pool or arena that has taken
// the whole device, or a host program that has handed every byte of HBM to
// its meshes, where a cudaMalloc would fail or steal memory the pool owns.
// cg_pk_bins_noalloc bins a half spectrum they already hold in device memory
// using a fixed scratch array compiled into this library instead of any
// allocation.  The call is synchronous on the caller's stream: it copies the
// bin sums into the caller's host arrays and waits for them.
//
// Scratch: g_pk_scratch, a file-scope __device__ array of 3 x
// CG_PK_NOALLOC_MAX_BINS doubles (24 KiB), present on every GPU that loads
// the library until the process exits.  Host code cannot use the symbol as
// a device address; the address is looked up with cudaGetSymbolAddress on
// the first call made with a device current, and again whenever that
// device's context has changed since (after cudaDeviceReset, the old
// address no longer belongs to the current context).
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "../../include/colagpu.h"
#include "internal.h"

extern int cg_set_error_from_lpt(int code, const char* msg);

namespace {

static __device__ __align__(256) double g_pk_scratch[3 * CG_PK_NOALLOC_MAX_BINS];

constexpr int T = CG_THREADS;
constexpr int kMaxDevices = 64;
// per device: the scratch address and the id of the context it belongs to
double* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

// Id of the current context (unique for the life of the process), or 0 when
// the driver does not report one.  The runtime makes the primary context
// current before this is called (cudaGetDevice / cudaFree-free set-up).
unsigned long long current_context_id() {
  typedef CUresult (*GetCur)(CUcontext*);
  typedef CUresult (*GetId)(CUcontext, unsigned long long*);
  static GetCur get_cur = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetCur>(f);
  }();
  static GetId get_id = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<GetId>(f);
  }();
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Same binning as the PM power spectrum (pm_kernels.cu k_pk_bin), for the
// half-spectrum layout spec[kx][ky][kz], kz = 0..N/2 fastest.
__global__ void __launch_bounds__(T) k_pk_bin_xyz(const float2* __restrict__ spec, int N,
                                                  int nbins, int deconv,
                                                  double* __restrict__ acc) {
  extern __shared__ double sb[];
  for (int i = threadIdx.x; i < 3 * nbins; i += T) sb[i] = 0.0;
  __syncthreads();
  const int nh = N / 2 + 1;
  const size_t total = (size_t)N * N * nh;
  for (size_t t = (size_t)blockIdx.x * T + threadIdx.x; t < total; t += (size_t)gridDim.x * T) {
    const int kz = (int)(t % nh);
    const int j = (int)((t / nh) % N);
    const int i = (int)(t / ((size_t)nh * N));
    const int si = i <= N / 2 ? i : i - N;
    const int sj = j <= N / 2 ? j : j - N;
    const double nm = sqrt((double)si * si + (double)sj * sj + (double)kz * kz);
    const int b = (int)floor(nm + 0.5) - 1;
    if (b < 0 || b >= nbins) continue;
    const double w = (kz == 0 || kz == N / 2) ? 1.0 : 2.0;
    const float2 s = spec[t];
    double p = (double)s.x * s.x + (double)s.y * s.y;
    if (deconv) {
      double win = 1.0;
      const int ns[3] = {si, sj, kz};
      for (int a = 0; a < 3; a++) {
        if (ns[a] != 0) {
          const double x = M_PI * ns[a] / N;
          const double sc = sin(x) / x;
          win *= sc * sc;
        }
      }
      p /= win * win;
    }
    atomicAdd(&sb[b], w);
    atomicAdd(&sb[nbins + b], w * nm);
    atomicAdd(&sb[2 * nbins + b], w * p);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * nbins; i += T)
    if (sb[i] != 0.0) atomicAdd(&acc[i], sb[i]);
}

}  // namespace

extern "C" int cg_pk_bins_noalloc(const void* d_spec, int n, float boxsize, int nbins, int flags,
                                  double* k_out, double* pk_out, double* nmodes_out,
                                  long long np, void* stream) {
  if (!d_spec || !k_out || !pk_out || !nmodes_out || n < 2 || n % 2 || !(boxsize > 0.0f))
    return cg_set_error_from_lpt(CG_EINVAL, "cg_pk_bins_noalloc: bad arguments");
  if (nbins < 1 || nbins > CG_PK_NOALLOC_MAX_BINS) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "cg_pk_bins_noalloc: nbins=%d outside 1..%d (the fixed scratch holds %d bins)",
             nbins, CG_PK_NOALLOC_MAX_BINS, CG_PK_NOALLOC_MAX_BINS);
    return cg_set_error_from_lpt(CG_EINVAL, msg);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return cg_set_error_from_lpt(CG_ECUDA, "cg_pk_bins_noalloc: no current device");
  // set-up, once per device and context: the device address of the scratch.
  // cudaGetSymbolAddress also makes the runtime's context current, so the
  // context id is read after it on the first call.
  unsigned long long ctx = g_scratch_addr[dev] ? current_context_id() : 0;
  if (!g_scratch_addr[dev] || ctx != g_scratch_ctx[dev]) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_pk_scratch);
    if (e != cudaSuccess || !ptr)
      return cg_set_error_from_lpt(CG_ECUDA, "cg_pk_bins_noalloc: cudaGetSymbolAddress failed");
    g_scratch_addr[dev] = static_cast<double*>(ptr);
    g_scratch_ctx[dev] = current_context_id();
  }
  double* acc = g_scratch_addr[dev];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the scratch keeps the previous call's sums: clear what must start at 0
  e = cudaMemsetAsync(acc, 0, sizeof(double) * 3 * nbins, st);
  if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ECUDA, "cg_pk_bins_noalloc: memset");
  const int blocks = cg_grid((long long)n * n * (n / 2 + 1), 8);
  prof_mark(st, CG_ST_OTHER);
  k_pk_bin_xyz<<<blocks, T, sizeof(double) * 3 * nbins, st>>>(
      static_cast<const float2*>(d_spec), n, nbins, flags & CG_PK_DECONVOLVE_CIC, acc);
  e = cudaGetLastError();
  // sums straight into the caller's arrays: nmodes <- sum w, k <- sum w|n|,
  // pk <- sum w |delta|^2, then normalised in place
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(nmodes_out, acc, sizeof(double) * nbins, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(k_out, acc + nbins, sizeof(double) * nbins, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pk_out, acc + 2 * nbins, sizeof(double) * nbins, cudaMemcpyDeviceToHost,
                        st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cg_set_error_from_lpt(CG_ECUDA, "cg_pk_bins_noalloc: launch");
  const double N = n, L = boxsize;
  const double kf = 2.0 * M_PI / L, norm = L * L * L / (N * N * N * N * N * N);
  const double shot = (flags & CG_PK_SUBTRACT_SHOT) && np > 0 ? L * L * L / (double)np : 0.0;
  for (int b = 0; b < nbins; b++) {
    const double w = nmodes_out[b];
    k_out[b] = w > 0 ? kf * k_out[b] / w : 0.0;
    pk_out[b] = w > 0 ? norm * pk_out[b] / w - shot : 0.0;
  }
  return CG_OK;
}
