// mvr_noalloc.cu -- mvr_filter_noalloc: the candidate filter (IVF probe ->
// candidate set -> approximate scores -> shortlist) for one query, with its
// scratch memory in a fixed array compiled into the library instead of
// memory obtained from cudaMalloc.
//
// Who needs it: a caller that must not allocate device memory while it
// serves queries -- e.g. a search plugin embedded in a host process whose GPU
// memory is entirely reserved by that host's own pool allocator (a database
// or inference server that carves HBM up front), or a latency-critical caller
// for which cudaMalloc / cudaFree and their implicit device-wide
// synchronisation are not acceptable.  Such a caller passes its own device
// buffers for inputs and outputs; the call itself allocates nothing.
//
// Limits and sharing rules:
//  * the scratch array is sized for indexes of at most kNoAllocMaxItems
//    (262,144) docs and queries of at most 32 tokens; larger inputs are
//    rejected with MVR_ERR_INVALID_ARG;
//  * the array (about 11 MB) is part of the library image: every GPU that
//    loads libmvr holds it until the process exits;
//  * every call on a device, from any thread or stream, uses the same array,
//    which keeps the previous call's contents; each call clears the parts
//    that must start in a known state.  Calls whose work overlaps on the GPU
//    (concurrent streams, or threads that do not order their streams) race on
//    the array and produce garbage -- serialise them;
//  * the first call on a device performs the one-time set-up
//    (cudaGetSymbolAddress of the array with that device current); make that
//    first call before any stream capture.
#include "mvr.h"

#include <mutex>
#include <string>

#include "mvr_common.cuh"
#include "mvr_kernels.cuh"

namespace mvr {
const DevIndex *handle_index(const mvr_index *h, int *device);
int record_error(int code, const char *msg);
}

namespace {

constexpr uint32_t kNoAllocMaxItems = 1u << 18;
constexpr uint32_t kNoAllocRankStride = 32;  // query tokens per call <= 32
constexpr size_t kStampOff = 0;
constexpr size_t kRankOff = kStampOff + (size_t)kNoAllocMaxItems * 4;
constexpr size_t kKeyOff = kRankOff + (size_t)kNoAllocMaxItems * kNoAllocRankStride;
constexpr size_t kQoffOff = kKeyOff + (size_t)kNoAllocMaxItems * 8;
constexpr size_t kQstatOff = kQoffOff + 256;
constexpr size_t kScratchBytes = kQstatOff + 256;

// The scratch array itself (device memory of every GPU that loads libmvr).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

int fail(int code, const std::string &msg) { return mvr::record_error(code, msg.c_str()); }

}  // namespace

extern "C" int mvr_filter_noalloc(mvr_index *h, const uint32_t *d_probe_id,
                                  const float *d_probe_score, uint32_t nq,
                                  uint32_t nprobe, uint32_t probe_topk,
                                  uint32_t *d_short_id, float *d_short_approx,
                                  uint32_t *d_n_short, void *cuda_stream) {
  if (!h || !d_probe_id || !d_probe_score || !d_short_id || !d_short_approx || !d_n_short)
    return fail(MVR_ERR_INVALID_ARG, "mvr_filter_noalloc: null argument");
  int device = 0;
  const mvr::DevIndex *ix = mvr::handle_index(h, &device);
  if (ix->n_item > kNoAllocMaxItems)
    return fail(MVR_ERR_INVALID_ARG,
                "mvr_filter_noalloc: index has " + std::to_string(ix->n_item) +
                    " docs; the allocation-free filter supports at most " +
                    std::to_string(kNoAllocMaxItems));
  if (nq == 0 || nq > kNoAllocRankStride)
    return fail(MVR_ERR_INVALID_ARG, "mvr_filter_noalloc: query tokens must be in [1, 32], got " +
                                         std::to_string(nq));
  if (nprobe == 0 || nprobe > (uint32_t)mvr::kMaxProbe || nprobe > ix->n_centroid)
    return fail(MVR_ERR_INVALID_ARG, "mvr_filter_noalloc: nprobe out of range");
  if (probe_topk == 0 || probe_topk > (uint32_t)mvr::kMaxShort)
    return fail(MVR_ERR_INVALID_ARG, "mvr_filter_noalloc: probe_topk out of range");
  if (device < 0 || device >= kMaxDevices)
    return fail(MVR_ERR_UNSUPPORTED, "mvr_filter_noalloc: device ordinal out of range");

  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (cudaSetDevice(device) != cudaSuccess)
    return fail(MVR_ERR_CUDA, "mvr_filter_noalloc: cudaSetDevice failed");
  struct Restore {
    int d;
    ~Restore() { if (d >= 0) cudaSetDevice(d); }
  } restore{prev};

  unsigned char *base;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {  // one-time set-up on this device (it is current)
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(MVR_ERR_CUDA, std::string("mvr_filter_noalloc: cudaGetSymbolAddress: ") +
                                      cudaGetErrorString(e));
      g_scratch_ptr[device] = static_cast<unsigned char *>(p);
    }
    base = g_scratch_ptr[device];
  }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  const size_t n = ix->n_item;
  uint64_t *q_off = reinterpret_cast<uint64_t *>(base + kQoffOff);
  // state that must start known: stamps 0, rank bytes 0xff, q_off = {0, nq}
  cudaError_t e = cudaMemsetAsync(base + kStampOff, 0, n * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + kRankOff, 0xff, n * kNoAllocRankStride, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(q_off, 0, 2 * sizeof(uint64_t), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(reinterpret_cast<unsigned char *>(q_off + 1), (int)nq, 1, st);
  if (e != cudaSuccess)
    return fail(MVR_ERR_CUDA, std::string("mvr_filter_noalloc: ") + cudaGetErrorString(e));
  mvr::FilterScratch scr{reinterpret_cast<uint32_t *>(base + kStampOff), base + kRankOff,
                         reinterpret_cast<uint64_t *>(base + kKeyOff), ix->n_item,
                         kNoAllocRankStride};
  int launches = 0;
  e = mvr::launch_filter(*ix, d_probe_id, d_probe_score, nprobe, q_off, 1, probe_topk, scr, 1u,
                         d_short_id, d_short_approx, d_n_short,
                         reinterpret_cast<uint32_t *>(base + kQstatOff), st, &launches);
  if (e != cudaSuccess)
    return fail(MVR_ERR_CUDA, std::string("mvr_filter_noalloc: ") + cudaGetErrorString(e));
  return MVR_OK;
}
