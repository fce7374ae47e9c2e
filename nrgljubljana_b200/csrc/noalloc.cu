// noalloc.cu -- transform() (M += factor * A * O * B^T) that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host thread that must not stall the device
// (cudaMalloc and cudaFree may synchronise it), a plugin running inside a process whose
// device memory is already reserved by another allocator, or code that is not allowed to
// own device memory at all. For them, the intermediate T = O * B^T of this entry point
// lives in a file-scope device array of fixed size instead of the context workspace, and
// the GEMM descriptors travel as kernel parameters instead of a staged device buffer.
#include <cuda.h>

#include <cstdint>
#include <mutex>

#include "ctx.h"
#include "kernels.h"

namespace {

// Scratch for T (ka x cols). Every GPU that loads this library holds these
// NRG_NOALLOC_SCRATCH_DOUBLES doubles until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[NRG_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 128;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // id of the CUDA context the address belongs to

// Unique id of the calling thread's current CUDA context (cuCtxGetId, taken from the driver
// through the runtime), 0 when the driver does not offer it.
unsigned long long current_context_id() {
  using Fn = CUresult (*)(CUcontext, unsigned long long*);
  static Fn fn = []() -> Fn {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<Fn>(p);
    cudaGetLastError();
    return nullptr;
  }();
  unsigned long long id = 0;
  if (!fn || fn(nullptr, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array on device `dev` (which must be current). Host code
// only sees a host-side stand-in under the array's name, so the address is taken with
// cudaGetSymbolAddress at the first call on the device and cached; it is taken again when
// the device's context has changed since (after a cudaDeviceReset, the array lives at an
// address of the new context).
int scratch_on(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return nrg::fail(NRG_ERR_ARG, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return nrg::fail(NRG_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<double*>(p);
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return NRG_OK;
}

}  // namespace

extern "C" int nrg_transform_noalloc(double* M, int64_t ldm, const double* A, int64_t lda, const double* O,
                                     int64_t ldo, const double* B, int64_t ldb, int rows, int cols, int ka, int kb,
                                     double factor, void* stream) {
  if (rows < 0 || cols < 0 || ka < 0 || kb < 0) return nrg::fail(NRG_ERR_ARG, "negative size");
  if (rows == 0 || cols == 0 || ka == 0 || kb == 0) return NRG_OK;  // finite_size() checks of the reference
  if (!M || !A || !B) return nrg::fail(NRG_ERR_ARG, "null pointer");
  if (!O && ka != kb) return nrg::fail(NRG_ERR_ARG, "O = NULL needs ka == kb");
  // Leading dimensions: dense row-major operands only (the diagonal O of nrg_gemm3, ldo == 0,
  // is not offered here and is rejected with every other ldo < kb).
  if (ldm < cols) return nrg::fail(NRG_ERR_ARG, "ldm = %lld < cols = %d", (long long)ldm, cols);
  if (lda < ka) return nrg::fail(NRG_ERR_ARG, "lda = %lld < ka = %d", (long long)lda, ka);
  if (ldb < kb) return nrg::fail(NRG_ERR_ARG, "ldb = %lld < kb = %d", (long long)ldb, kb);
  if (O && ldo < kb)
    return nrg::fail(NRG_ERR_ARG, "ldo = %lld < kb = %d (a diagonal O, ldo = 0, needs nrg_gemm3_batch)",
                     (long long)ldo, kb);
  if (!(factor == factor) || factor - factor != 0.0) return nrg::fail(NRG_ERR_ARG, "non-finite factor");
  if (O && (size_t)ka * (size_t)cols > (size_t)NRG_NOALLOC_SCRATCH_DOUBLES)
    return nrg::fail(NRG_ERR_ARG,
                     "ka * cols = %lld exceeds the static scratch of %d doubles of nrg_transform_noalloc",
                     (long long)ka * cols, NRG_NOALLOC_SCRATCH_DOUBLES);
  auto s = static_cast<cudaStream_t>(stream);
  const double* Bm = B;
  int64_t ldbm = ldb;
  int transB = 1;
  if (O) {
    int dev = 0;
    NRG_CK(cudaGetDevice(&dev));
    double* T = nullptr;
    const int rc = scratch_on(dev, &T);
    if (rc) return rc;
    // T = O * B^T (ka x cols), fully overwritten (beta = 0): no clearing is needed.
    nrg::GemmOut o1{};
    o1.C = T;
    o1.ldc = cols;
    o1.M = ka;
    o1.N = cols;
    o1.beta = 0.0;
    nrg::GemmSeg g1{};
    g1.A = O;
    g1.lda = ldo;
    g1.B = B;
    g1.ldb = ldb;
    g1.K = kb;
    g1.transB = 1;
    g1.alpha = 1.0;
    NRG_CK(nrg::gemm_one_launch(o1, g1, s));
    Bm = T;
    ldbm = cols;
    transB = 0;
  }
  // M += factor * A * T   (or factor * A * B^T when O is the identity)
  nrg::GemmOut o2{};
  o2.C = M;
  o2.ldc = ldm;
  o2.M = rows;
  o2.N = cols;
  o2.beta = 1.0;
  nrg::GemmSeg g2{};
  g2.A = A;
  g2.lda = lda;
  g2.B = Bm;
  g2.ldb = ldbm;
  g2.K = ka;
  g2.transB = transB;
  g2.alpha = factor;
  NRG_CK(nrg::gemm_one_launch(o2, g2, s));
  return NRG_OK;
}
