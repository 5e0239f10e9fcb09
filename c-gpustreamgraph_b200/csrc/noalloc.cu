// noalloc.cu -- sgs_sssp_csr_noalloc: a from-scratch SSSP/BFS over a CSR that
// the caller already holds in device memory, for callers that cannot allocate
// device memory themselves: code running inside an allocator hook or a memory
// pool callback (an allocation there would re-enter the allocator), and
// embedders whose memory is fixed at start-up (real-time or safety builds that
// forbid cudaMalloc after initialisation).
//
// It runs the same relaxation kernel (seg_map) as the engine's SSSP/BFS
// queries, but its scratch -- packed (value,parent) state, round stamps, the
// two frontier buffers and the round counters -- lives in one file-scope
// static __device__ array of fixed size instead of memory from cudaMalloc.
// The library therefore reserves that array (about 36 MB) on every GPU where
// it is loaded, until the process exits.
//
// The array is shared by all calls on a device and keeps whatever the last
// call left in it; each call clears the parts that must start at zero.  Two
// calls whose work overlaps on the GPU (different streams, or different host
// threads on one device) race on the array and give wrong results: serialise
// them.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture begins.  The address is cached per device ordinal
// for the life of the process: after a cudaDeviceReset the cached address no
// longer names the array, so the entry point must not be used on that device
// again in the same process.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/sgs.h"
#include "sgs_segmap.cuh"

namespace sgs {
void set_last_error(const std::string &msg);
}

namespace {

using namespace sgs;

constexpr uint32_t NA_MAX_NV = SGS_NOALLOC_MAX_VERTICES;
constexpr uint64_t NA_MAX_E = SGS_NOALLOC_MAX_EDGES;
constexpr uint32_t NA_UNITS = (uint32_t)((NA_MAX_E + 3ull * NA_MAX_NV) / UNIT + 2);
constexpr uint32_t NA_MAX_ROUNDS = 1000;  // the engine's default round limit
constexpr uint32_t NA_BATCH = 16;

// Byte offsets of the scratch regions (each 256-B aligned).
constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t OFF_ST = 0;
constexpr size_t OFF_MARK = al(OFF_ST + sizeof(unsigned long long) * NA_MAX_NV);
constexpr size_t OFF_VTX0 = al(OFF_MARK + sizeof(uint32_t) * NA_MAX_NV);
constexpr size_t OFF_VTX1 = al(OFF_VTX0 + sizeof(uint32_t) * NA_MAX_NV);
constexpr size_t OFF_EB0 = al(OFF_VTX1 + sizeof(uint32_t) * NA_MAX_NV);
constexpr size_t OFF_EB1 = al(OFF_EB0 + sizeof(uint64_t) * NA_MAX_NV);
constexpr size_t OFF_LEN0 = al(OFF_EB1 + sizeof(uint64_t) * NA_MAX_NV);
constexpr size_t OFF_LEN1 = al(OFF_LEN0 + sizeof(uint32_t) * NA_MAX_NV);
constexpr size_t OFF_US0 = al(OFF_LEN1 + sizeof(uint32_t) * NA_MAX_NV);
constexpr size_t OFF_US1 = al(OFF_US0 + sizeof(uint32_t) * NA_UNITS);
constexpr size_t OFF_CNT = al(OFF_US1 + sizeof(uint32_t) * NA_UNITS);
constexpr size_t OFF_ERR = al(OFF_CNT + sizeof(unsigned long long) * (NA_MAX_ROUNDS + 2));
constexpr size_t NA_BYTES = al(OFF_ERR + sizeof(unsigned int) * 4);

// The scratch: fixed size, file scope, one per device context.
static __device__ __align__(256) unsigned char g_na_scratch[NA_BYTES];

std::mutex g_na_mu;
void *g_na_ptr[64] = {};  // per device ordinal: device address of g_na_scratch

struct NaFail {
  int code;
  std::string msg;
};

struct CsrPay {
  uint64_t off;
  uint32_t val;
  uint32_t pad;
};

// SSSP/BFS relaxation over a plain CSR: the same packed (value,parent)
// atomicMin as the engine's RelaxMinOp, so the result (values and
// smallest-id tight parents) is identical.  Out-of-range destinations and
// zero weights are recorded in err and skipped.
struct CsrRelaxOp {
  static constexpr bool kAppends = true;
  static constexpr bool kQuad = false;
  using Payload = CsrPay;
  const uint64_t *row;
  const uint32_t *col;
  const uint32_t *w;  // null: unit weights (BFS)
  unsigned long long *st;
  uint32_t *mark;
  unsigned int *err;
  uint32_t nv;
  uint32_t stamp;
  __device__ __forceinline__ Payload load(uint32_t, uint32_t v) const {
    CsrPay p;
    p.off = row[v];
    p.val = (uint32_t)(__ldcg(&st[v]) >> 32);
    p.pad = 0;
    return p;
  }
  __device__ __forceinline__ uint32_t visit(uint32_t u, const Payload &p, uint32_t j, bool &app,
                                            uint32_t &av, uint32_t &ad) const {
    const uint32_t dst = col[p.off + j];
    if (dst >= nv) { atomicOr(err, 1u); return 0; }
    if (p.val == INF32) return 1;
    const uint32_t wt = w ? w[p.off + j] : 1u;
    if (wt == 0) { atomicOr(err, 2u); return 1; }
    const uint64_t nd = (uint64_t)p.val + wt;
    if (nd >= INF32) return 1;
    const unsigned long long np = ((unsigned long long)nd << 32) | u;
    if (np >= __ldcg(&st[dst])) return 1;
    const unsigned long long old = atomicMin(&st[dst], np);
    if (nd < (old >> 32)) {
      if (__ldcg(&mark[dst]) != stamp && atomicExch(&mark[dst], stamp) != stamp) {
        const uint32_t d = (uint32_t)(row[dst + 1] - row[dst]);
        if (d) { app = true; av = dst; ad = d; }
      }
    }
    return 1;
  }
};

__global__ void k_na_init(unsigned long long *st, uint32_t nv, uint32_t src, const uint64_t *row,
                          unsigned int *err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    st[v] = (v == src) ? (unsigned long long)INF32 : ~0ull;
    if (row[v + 1] < row[v]) atomicOr(err, 4u);
  }
}

__global__ void k_na_seed(FrontierView out, const uint64_t *row, uint32_t src) {
  if (threadIdx.x >= 32) return;
  const uint32_t d = (uint32_t)(row[src + 1] - row[src]);
  frontier_append(out, threadIdx.x == 0 && d > 0, src, d);
}

__global__ void k_na_split(const unsigned long long *st, uint32_t nv, uint32_t *val, uint32_t *par) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += stride) {
    const unsigned long long s = st[v];
    if (val) val[v] = (uint32_t)(s >> 32);
    if (par) par[v] = (uint32_t)s;
  }
}

void ck(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw NaFail{SGS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}
#define NACK(x) ck((x), #x)

// Device address of the scratch array for the current device (looked up once
// per device, with that device current).
unsigned char *scratch_for_current_device() {
  int dev = 0;
  NACK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw NaFail{SGS_ERR_INVALID, "device ordinal out of range"};
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    NACK(cudaGetSymbolAddress(&p, g_na_scratch));
    g_na_ptr[dev] = p;
  }
  return (unsigned char *)g_na_ptr[dev];
}

void run(uint32_t nv, const uint64_t *row, const uint32_t *col, const uint32_t *w, uint32_t source,
         uint32_t *dist, uint32_t *parent, cudaStream_t s) {
  if (nv == 0 || nv > NA_MAX_NV)
    throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: nv must be in [1, " +
                                      std::to_string(NA_MAX_NV) + "]"};
  if (!row || !col || !dist) throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: null pointer"};
  unsigned char *base = scratch_for_current_device();
  uint64_t ne = 0;
  NACK(cudaMemcpyAsync(&ne, row + nv, sizeof(ne), cudaMemcpyDeviceToHost, s));
  NACK(cudaStreamSynchronize(s));
  if (ne > NA_MAX_E)
    throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: more than " + std::to_string(NA_MAX_E) +
                                      " edges"};
  source = source < nv ? source : nv - 1;  // clamped like the engine's queries
  auto *st = (unsigned long long *)(base + OFF_ST);
  auto *mark = (uint32_t *)(base + OFF_MARK);
  auto *cnt = (unsigned long long *)(base + OFF_CNT);
  auto *err = (unsigned int *)(base + OFF_ERR);
  FrontierView f[2];
  f[0].vtx = (uint32_t *)(base + OFF_VTX0);
  f[1].vtx = (uint32_t *)(base + OFF_VTX1);
  f[0].ebase = (uint64_t *)(base + OFF_EB0);
  f[1].ebase = (uint64_t *)(base + OFF_EB1);
  f[0].len = (uint32_t *)(base + OFF_LEN0);
  f[1].len = (uint32_t *)(base + OFF_LEN1);
  f[0].ustart = (uint32_t *)(base + OFF_US0);
  f[1].ustart = (uint32_t *)(base + OFF_US1);
  f[0].ucap = f[1].ucap = NA_UNITS;
  // clear what must start at zero: counters, error word, stamps
  NACK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * (NA_MAX_ROUNDS + 2), s));
  NACK(cudaMemsetAsync(err, 0, sizeof(unsigned int), s));
  NACK(cudaMemsetAsync(mark, 0, sizeof(uint32_t) * nv, s));
  int nsm = 148, dev = 0;
  NACK(cudaGetDevice(&dev));
  NACK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const uint32_t grid = (uint32_t)nsm * 8;
  const uint32_t egrid = (uint32_t)std::min<uint64_t>((nv + 255) / 256, (uint64_t)grid);
  k_na_init<<<egrid, 256, 0, s>>>(st, nv, source, row, err);
  NACK(cudaGetLastError());
  {
    // reject decreasing row offsets before any kernel indexes col with them
    unsigned int e0 = 0;
    uint64_t r0 = 0;
    NACK(cudaMemcpyAsync(&e0, err, sizeof(e0), cudaMemcpyDeviceToHost, s));
    NACK(cudaMemcpyAsync(&r0, row, sizeof(r0), cudaMemcpyDeviceToHost, s));
    NACK(cudaStreamSynchronize(s));
    if (e0 & 4u || r0 != 0)
      throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: row offsets must start at 0 and not decrease"};
  }
  f[0].counter = (uint64_t *)cnt;
  k_na_seed<<<1, 32, 0, s>>>(f[0], row, source);
  NACK(cudaGetLastError());
  unsigned long long h[NA_BATCH + 1];
  uint32_t r = 0, rb = 2;
  bool done = false;
  while (r < NA_MAX_ROUNDS && !done) {
    const uint32_t nb = std::min(rb, NA_MAX_ROUNDS - r);
    for (uint32_t k = 0; k < nb; ++k) {
      const uint32_t rr = r + k;
      FrontierView in = f[rr & 1], out = f[(rr + 1) & 1];
      in.counter = (uint64_t *)(cnt + rr);
      out.counter = (uint64_t *)(cnt + rr + 1);
      CsrRelaxOp op{row, col, w, st, mark, err, nv, rr + 1};
      seg_map<<<grid, RELAX_THREADS, 0, s>>>(in, out, op, nullptr);
    }
    NACK(cudaGetLastError());
    NACK(cudaMemcpyAsync(h, cnt + r + 1, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, s));
    NACK(cudaStreamSynchronize(s));
    for (uint32_t k = 0; k < nb && !done; ++k) done = h[k] == 0;
    r += nb;
    rb = std::min<uint32_t>(rb * 2, NA_BATCH);
  }
  unsigned int herr = 0;
  NACK(cudaMemcpyAsync(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost, s));
  NACK(cudaStreamSynchronize(s));
  if (herr & 1u) throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: edge destination >= nv"};
  if (herr & 2u) throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: weight 0 (weights must be >= 1)"};
  if (herr & 4u) throw NaFail{SGS_ERR_INVALID, "sgs_sssp_csr_noalloc: row offsets decrease"};
  if (!done) throw NaFail{SGS_ERR_NOCONV, "sgs_sssp_csr_noalloc: round limit reached"};
  k_na_split<<<egrid, 256, 0, s>>>(st, nv, dist, parent);
  NACK(cudaGetLastError());
  NACK(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" SGS_API int sgs_sssp_csr_noalloc(uint32_t nv, const uint64_t *row, const uint32_t *col,
                                            const uint32_t *w, uint32_t source, uint32_t *dist,
                                            uint32_t *parent, void *stream) {
  try {
    run(nv, row, col, w, source, dist, parent, (cudaStream_t)stream);
    return SGS_OK;
  } catch (const NaFail &f) {
    sgs::set_last_error(f.msg);
    return f.code;
  }
}
