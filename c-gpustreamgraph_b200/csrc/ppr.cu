// ppr.cu -- weighted (personalized) PageRank with a hand-written adjoint.
//
// Fixed point (the reference's unnormalised PageRank of
// samples/hybrid_pr/hybrid_pr.cu:26-151 generalised to edge weights and
// teleport vectors): for each of K teleport vectors t_k,
//     x_k = (1 - alpha) t_k + alpha P^T x_k,   P[u,v] = w_uv / s_u, s_u = sum_v w_uv
// (rows without out-edges drop their mass, as in the reference).  With
// t_k = 1 and unit weights this is exactly the reference's PageRank.
//
// Adjoint for an upstream gradient G = dL/dX:
//     Y = G + alpha P Y                       (transposed fixed point)
//     dL/dT = (1 - alpha) Y
//     dL/dw_uv = (1/s_u) sum_k X[u,k] (alpha Y[v,k] - Y[u,k] + G[u,k])
// (the derivative of the row normalisation included; parallel edges each get
// the same term).  All state is FP64, vertex-major [nv][K], so the K values of
// one vertex are one contiguous row of 8K bytes.
//
// Both fixed points are Jacobi iterations of one gather,
//     out[v,:] = c B[v,:] + alpha sum_{i in adj(v)} p_i x[nbr_i, :]
// over the CSC (forward: in-edges) or the CSR (adjoint: out-edges), with the
// edge probabilities p = P[u,v] precomputed once per weight vector.
//
// Work split: a warp owns a work item.  Vertices of degree <= PIECE are one
// item each; a heavier vertex (R-MAT hubs reach 10^5 in-edges) is cut into
// pieces of PIECE edges whose partial sums go to a scratch row each and are
// added up, in piece order, by a finalize kernel -- so no warp walks more
// than PIECE edges and the sums are deterministic.  Inside a warp, LPE lanes
// cover the columns of one neighbour row (CPL columns per lane) and 32/LPE
// neighbours are gathered at once, four deep, so one neighbour row is one
// coalesced read for any K.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/sgs.h"

namespace sgs {
void set_last_error(const std::string &msg);
}

namespace {

struct PprFail {
  int code;
  std::string msg;
};

void ck(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return;
  cudaGetLastError();
  throw PprFail{e == cudaErrorMemoryAllocation ? SGS_ERR_OOM : SGS_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e)};
}
#define PCK(x) ck((x), #x)

template <class T>
struct Buf {
  T *p = nullptr;
  size_t n = 0;
  void ensure(size_t want) {
    want = std::max<size_t>(want, 1);
    if (p && want <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    PCK(cudaMalloc((void **)&p, want * sizeof(T)));
    n = want;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

constexpr int THREADS = 256;
constexpr uint32_t PIECE = 256;  // most edges one warp walks per item

__device__ __forceinline__ uint32_t warp_id() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint32_t num_warps() { return (gridDim.x * blockDim.x) >> 5; }

__global__ void k_validate(const uint64_t *row, const uint32_t *col, uint32_t nv, uint64_t ne,
                           unsigned int *err) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0 && row[0] != 0) atomicOr(err, 2u);
  for (uint64_t v = tid; v < nv; v += stride)
    if (row[v + 1] < row[v]) atomicOr(err, 2u);
  for (uint64_t i = tid; i < ne; i += stride)
    if (col[i] >= nv) atomicOr(err, 1u);
}

__global__ void k_edge_src(const uint64_t *row, uint32_t nv, uint32_t *src) {
  const int lane = threadIdx.x & 31;
  for (uint32_t u = warp_id(); u < nv; u += num_warps())
    for (uint64_t e = row[u] + lane; e < row[u + 1]; e += 32) src[e] = u;
}

__global__ void k_iota(uint32_t *a, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = (uint32_t)i;
}

// crow[v] = first position of destination >= v in the sorted destinations.
__global__ void k_csc_rows(const uint32_t *sorted_dst, uint64_t ne, uint32_t nv, uint64_t *crow) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t l = 0, r = ne;
    while (l < r) {
      const uint64_t m = (l + r) >> 1;
      if (sorted_dst[m] < v) l = m + 1;
      else r = m;
    }
    crow[v] = l;
  }
}

__global__ void k_gather_u32(const uint32_t *a, const uint32_t *idx, uint64_t n, uint32_t *b) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = a[idx[i]];
}

// cnt[v] = number of pieces of v (0 for a vertex of degree <= PIECE); cnt[nv] = 0.
__global__ void k_piece_count(const uint64_t *ptr, uint32_t nv, uint32_t *cnt) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v <= nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t d = v < nv ? ptr[v + 1] - ptr[v] : 0;
    cnt[v] = d > PIECE ? (uint32_t)((d + PIECE - 1) / PIECE) : 0u;
  }
}

// pv[poff[v] + j] = v for each piece j of v.
__global__ void k_piece_fill(const uint32_t *poff, uint32_t nv, uint32_t *pv) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x)
    for (uint32_t p = poff[v]; p < poff[v + 1]; ++p) pv[p] = (uint32_t)v;
}

// inv_s[u] = 1 / sum of u's out-edge weights (0 without out-edges), and the
// CSR edge probabilities pr[e] = w[e] inv_s[u].  err bit 0: a weight that is
// not positive and finite.
__global__ void k_row_probs(const uint64_t *row, uint32_t nv, const double *w, double *inv_s,
                            double *pr, unsigned int *err) {
  const int lane = threadIdx.x & 31;
  for (uint32_t u = warp_id(); u < nv; u += num_warps()) {
    double s = 0.0;
    for (uint64_t e = row[u] + lane; e < row[u + 1]; e += 32) {
      const double x = w[e];
      if (!(x > 0.0) || !isfinite(x)) atomicOr(err, 1u);
      s += x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    const double is = s > 0.0 ? 1.0 / s : 0.0;
    if (lane == 0) inv_s[u] = is;
    for (uint64_t e = row[u] + lane; e < row[u + 1]; e += 32) pr[e] = w[e] * is;
  }
}

// CSC probabilities: pc[i] = pr[ceid[i]].
__global__ void k_csc_probs(const double *pr, const uint32_t *ceid, uint64_t ne, double *pc) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne;
       i += (uint64_t)gridDim.x * blockDim.x)
    pc[i] = pr[ceid[i]];
}

// Narrow rows (K < 32): each lane group loads its own neighbours' ids,
// probabilities and rows, four neighbours deep (neighbours b+eg, b+eg+NEG, ...).
template <int LPE, int CPL>
__device__ __forceinline__ void gather_rows_direct(const uint32_t *__restrict__ nbr,
                                                   const double *__restrict__ p, uint64_t b,
                                                   uint64_t e, int eg, uint32_t kb, uint32_t K,
                                                   const double *__restrict__ x,
                                                   double (&acc)[CPL]) {
  constexpr int NEG = 32 / LPE;
  uint64_t i = b + eg;
  for (; i + 3 * NEG < e; i += 4 * NEG) {
    uint32_t u[4];
    double pp[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      u[q] = nbr[i + q * NEG];
      pp[q] = p[i + q * NEG];
    }
    double xv[4][CPL];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int j = 0; j < CPL; ++j) {
        const uint32_t k = kb + j * LPE;
        xv[q][j] = k < K ? x[(uint64_t)u[q] * K + k] : 0.0;
      }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int j = 0; j < CPL; ++j) acc[j] = fma(pp[q], xv[q][j], acc[j]);
  }
  for (; i < e; i += NEG) {
    const uint32_t u = nbr[i];
    const double pp = p[i];
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
      const uint32_t k = kb + j * LPE;
      if (k < K) acc[j] = fma(pp, x[(uint64_t)u * K + k], acc[j]);
    }
  }
}

// acc[j] += sum_{i in [b,e)} p[i] x[nbr[i], kb + j LPE] for this lane's
// neighbour group eg.  Neighbour ids and probabilities come 32 at a time in
// one coalesced load per warp and are handed to the lane groups by shuffles
// (group eg takes neighbours eg, eg + NEG, ...), so the only dependent load
// per neighbour is its row; DEPTH neighbours per group are in flight at once.
template <int LPE, int CPL>
__device__ __forceinline__ void gather_rows(const uint32_t *__restrict__ nbr,
                                            const double *__restrict__ p, uint64_t b, uint64_t e,
                                            int lane, int eg, uint32_t kb, uint32_t K,
                                            const double *__restrict__ x, double (&acc)[CPL]) {
  constexpr int NEG = 32 / LPE;
  constexpr int DEPTH = LPE < 4 ? LPE : 4;
  for (uint64_t c = b; c < e; c += 32) {
    const uint32_t cnt = e - c < 32 ? (uint32_t)(e - c) : 32u;
    const uint32_t mu = (uint32_t)lane < cnt ? __ldg(nbr + c + lane) : 0u;
    const double mp = (uint32_t)lane < cnt ? __ldg(p + c + lane) : 0.0;
#pragma unroll 1
    for (int r0 = 0; r0 < LPE && (uint32_t)(NEG * r0) < cnt; r0 += DEPTH) {
      uint32_t u[DEPTH];
      double pp[DEPTH];
      bool ok[DEPTH];
#pragma unroll
      for (int q = 0; q < DEPTH; ++q) {
        const int jn = eg + NEG * (r0 + q);  // < 32
        u[q] = __shfl_sync(0xFFFFFFFFu, mu, jn);
        pp[q] = __shfl_sync(0xFFFFFFFFu, mp, jn);
        ok[q] = (uint32_t)jn < cnt;
      }
      double xv[DEPTH][CPL];
#pragma unroll
      for (int q = 0; q < DEPTH; ++q)
#pragma unroll
        for (int jj = 0; jj < CPL; ++jj) {
          const uint32_t k = kb + jj * LPE;
          xv[q][jj] = ok[q] && k < K ? __ldg(x + (uint64_t)u[q] * K + k) : 0.0;
        }
#pragma unroll
      for (int q = 0; q < DEPTH; ++q)
#pragma unroll
        for (int jj = 0; jj < CPL; ++jj) acc[jj] = fma(pp[q], xv[q][jj], acc[jj]);
    }
  }
}

// One Jacobi step over the work items [0, npieces) (pieces of heavy vertices:
// partial sums to part[piece][K]) and [npieces, npieces + nv) (light vertices:
// out[v,k] = c B[v,k] + alpha sum p x, |out - x| added to *diff).
template <int LPE, int CPL>
__global__ void __launch_bounds__(THREADS, LPE == 32 ? 1 : 8)
    k_ppr_step(const uint64_t *__restrict__ ptr, const uint32_t *__restrict__ nbr,
               const double *__restrict__ p, uint32_t nv, const uint32_t *__restrict__ pv,
               const uint32_t *__restrict__ poff, uint32_t npieces, uint32_t K, double alpha,
               double c, const double *__restrict__ B, const double *__restrict__ x,
               double *__restrict__ out, double *__restrict__ part, double *diff) {
  const int lane = threadIdx.x & 31;
  const int sub = lane % LPE, eg = lane / LPE;
  double dsum = 0.0;
  const uint32_t items = npieces + nv;
  const uint32_t W = num_warps();
  uint64_t pb = 0, pe = 0;  // bounds of this warp's next light vertex, loaded ahead
  bool have = false;
  for (uint32_t wi = warp_id(); wi < items; wi += W) {
    uint32_t v;
    uint64_t b, e;
    const bool piece = wi < npieces;
    if (piece) {
      v = pv[wi];
      b = ptr[v] + (uint64_t)(wi - poff[v]) * PIECE;
      e = min(b + PIECE, ptr[v + 1]);
    } else {
      v = wi - npieces;
      if (have) {
        b = pb;
        e = pe;
      } else {
        b = ptr[v];
        e = ptr[v + 1];
      }
      if constexpr (LPE == 32) {  // the narrow forms have no registers to spare
        have = wi + W < items;
        if (have) {
          pb = ptr[v + W];
          pe = ptr[v + W + 1];
        }
      }
      if (e - b > PIECE) continue;  // summed by its pieces
    }
    for (uint32_t k0 = 0; k0 < K; k0 += LPE * CPL) {
      double acc[CPL];
#pragma unroll
      for (int j = 0; j < CPL; ++j) acc[j] = 0.0;
      if constexpr (LPE == 32)
        gather_rows<LPE, CPL>(nbr, p, b, e, lane, eg, k0 + sub, K, x, acc);
      else
        gather_rows_direct<LPE, CPL>(nbr, p, b, e, eg, k0 + sub, K, x, acc);
#pragma unroll
      for (int j = 0; j < CPL; ++j)
#pragma unroll
        for (int o = 16; o >= LPE; o >>= 1) acc[j] += __shfl_xor_sync(0xFFFFFFFFu, acc[j], o);
      if (eg == 0) {
#pragma unroll
        for (int j = 0; j < CPL; ++j) {
          const uint32_t k = k0 + sub + j * LPE;
          if (k >= K) continue;
          if (piece) {
            part[(uint64_t)wi * K + k] = acc[j];
          } else {
            const uint64_t o = (uint64_t)v * K + k;
            const double nx = c * B[o] + alpha * acc[j];
            dsum += fabs(nx - x[o]);
            out[o] = nx;
          }
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xFFFFFFFFu, dsum, o);
  if (lane == 0 && dsum != 0.0) atomicAdd(diff, dsum);
}

// Heavy vertices: out[v,k] = c B[v,k] + alpha (sum of v's piece rows, in
// piece order); one warp per first piece.
__global__ void __launch_bounds__(THREADS)
    k_ppr_finalize(const uint32_t *__restrict__ pv, const uint32_t *__restrict__ poff,
                   uint32_t npieces, uint32_t K, double alpha, double c,
                   const double *__restrict__ B, const double *__restrict__ x,
                   double *__restrict__ out, const double *__restrict__ part, double *diff) {
  const int lane = threadIdx.x & 31;
  double dsum = 0.0;
  for (uint32_t pi = warp_id(); pi < npieces; pi += num_warps()) {
    const uint32_t v = pv[pi];
    if (poff[v] != pi) continue;
    const uint32_t pe = poff[v + 1];
    for (uint32_t k = lane; k < K; k += 32) {
      double s = 0.0;
      for (uint32_t q = pi; q < pe; ++q) s += part[(uint64_t)q * K + k];
      const uint64_t o = (uint64_t)v * K + k;
      const double nx = c * B[o] + alpha * s;
      dsum += fabs(nx - x[o]);
      out[o] = nx;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xFFFFFFFFu, dsum, o);
  if (lane == 0 && dsum != 0.0) atomicAdd(diff, dsum);
}

// gw[e] = inv_s[u] (alpha sum_k X[u,k] Y[v,k] + c_u) for e = (u,v), where
// c_u = sum_k X[u,k] (G[u,k] - Y[u,k]); work items as in k_ppr_step over the
// CSR (each item recomputes c_u for its source).
template <int LPE>
__global__ void __launch_bounds__(THREADS)
    k_ppr_edge_grad(const uint64_t *__restrict__ row, const uint32_t *__restrict__ col,
                    const double *__restrict__ inv_s, uint32_t nv, const uint32_t *__restrict__ pv,
                    const uint32_t *__restrict__ poff, uint32_t npieces, uint32_t K, double alpha,
                    const double *__restrict__ X, const double *__restrict__ Y,
                    const double *__restrict__ G, double *__restrict__ gw) {
  constexpr int NEG = 32 / LPE;
  const int lane = threadIdx.x & 31;
  const int sub = lane % LPE, eg = lane / LPE;
  const uint32_t items = npieces + nv;
  for (uint32_t wi = warp_id(); wi < items; wi += num_warps()) {
    uint32_t u;
    uint64_t b, e;
    if (wi < npieces) {
      u = pv[wi];
      b = row[u] + (uint64_t)(wi - poff[u]) * PIECE;
      e = min(b + PIECE, row[u + 1]);
    } else {
      u = wi - npieces;
      b = row[u];
      e = row[u + 1];
      if (e == b || e - b > PIECE) continue;
    }
    const uint64_t ou = (uint64_t)u * K;
    double cu = 0.0;
    for (uint32_t k = lane; k < K; k += 32) cu += X[ou + k] * (G[ou + k] - Y[ou + k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cu += __shfl_xor_sync(0xFFFFFFFFu, cu, o);
    const double is = inv_s[u];
    for (uint64_t e0 = b; e0 < e; e0 += NEG) {
      const uint64_t i = e0 + eg;
      const bool ok = i < e;
      const uint32_t v = ok ? col[i] : 0u;
      double t = 0.0;
      if (ok)
        for (uint32_t k = sub; k < K; k += LPE) t = fma(X[ou + k], Y[(uint64_t)v * K + k], t);
#pragma unroll
      for (int o = LPE / 2; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
      if (ok && sub == 0) gw[i] = is * fma(alpha, t, cu);
    }
  }
}

__global__ void k_scale(const double *a, double s, uint64_t n, double *b) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = s * a[i];
}

int lanes_per_edge(uint32_t K) {
  int l = 1;
  while (l < 32 && (uint32_t)l < K) l <<= 1;
  return l;
}

// The edge lists of one direction with their heavy-vertex pieces.
struct Adj {
  const uint64_t *ptr = nullptr;
  const uint32_t *nbr = nullptr;
  Buf<uint32_t> poff, pv;
  uint32_t npieces = 0;
};

}  // namespace

// A graph prepared for PPR: the CSR (out-edges) and a CSC (in-edges) whose
// entries carry the CSR index of the edge, so weights given in CSR order
// apply to both directions.
struct sgs_ppr {
  int dev = 0;
  int nsm = 148;
  cudaStream_t s = nullptr;
  uint32_t nv = 0;
  uint64_t ne = 0;
  Buf<uint64_t> row, crow;
  Buf<uint32_t> col, csrc, ceid;
  Buf<double> w, inv_s, pr, pc, t, x, xn, g, y, yn, part, diff;
  Buf<unsigned int> err;
  Adj in, out;  // CSC (forward) and CSR (adjoint, edge gradient)
  // timing and counters
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // 2 per step of a batch (timing on)
  cudaEvent_t call_ev[2] = {nullptr, nullptr};
  sgs_ppr_stats st{};
  uint64_t n_launch = 0;
  ~sgs_ppr() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    for (cudaEvent_t e : call_ev)
      if (e) cudaEventDestroy(e);
    if (s) cudaStreamDestroy(s);
  }
  void events() {
    if (!call_ev[0]) {
      PCK(cudaEventCreate(&call_ev[0]));
      PCK(cudaEventCreate(&call_ev[1]));
    }
    while (ev.size() < 64) {
      cudaEvent_t e;
      PCK(cudaEventCreate(&e));
      ev.push_back(e);
    }
  }
  // begin/end of a public call: device time of everything on the stream
  void call_begin() {
    events();
    st.iters = 0;
    st.steps_ms = 0.0;
    st.ms = 0.0;
    PCK(cudaEventRecord(call_ev[0], s));
  }
  void call_end() {
    PCK(cudaEventRecord(call_ev[1], s));
    PCK(cudaEventSynchronize(call_ev[1]));
    float ms = 0.f;
    PCK(cudaEventElapsedTime(&ms, call_ev[0], call_ev[1]));
    st.ms = ms;
    st.kernel_launches = n_launch;
  }
  uint32_t grid() const { return (uint32_t)nsm * 8; }
  // One wave: every block resident at once, so the grid-stride split of the
  // work items has no second partial wave.
  std::map<const void *, uint32_t> rgrid_cache;
  uint32_t rgrid(const void *f) {
    auto it = rgrid_cache.find(f);
    if (it != rgrid_cache.end()) return it->second;
    int b = 0;
    PCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, THREADS, 0));
    const uint32_t g = (uint32_t)nsm * (uint32_t)std::max(b, 1);
    rgrid_cache[f] = g;
    return g;
  }
  void sync() { PCK(cudaStreamSynchronize(s)); }
  // algorithmic bytes of one Jacobi step with K columns: per edge the 4-B
  // neighbour id, the 8-B probability and the neighbour's 8K-B row; per
  // vertex two 8-B offsets and 8K B each of B and x read and out written
  double step_bytes(uint32_t K) const {
    return (double)ne * (12.0 + 8.0 * K) + (double)nv * (16.0 + 24.0 * K);
  }
  cudaMemcpyKind kin(int mem) const {
    return mem == SGS_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  }
  cudaMemcpyKind kout(int mem) const {
    return mem == SGS_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  }

  void pieces(Adj &a, const uint64_t *ptr, const uint32_t *nbr) {
    a.ptr = ptr;
    a.nbr = nbr;
    a.poff.ensure((size_t)nv + 1);
    { ++n_launch; k_piece_count<<<grid(), THREADS, 0, s>>>(ptr, nv, a.poff.p); }
    size_t tb = 0;
    PCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, a.poff.p, a.poff.p, (int)(nv + 1), s));
    Buf<unsigned char> tmp;
    tmp.ensure(tb);
    PCK(cub::DeviceScan::ExclusiveSum(tmp.p, tb, a.poff.p, a.poff.p, (int)(nv + 1), s));
    PCK(cudaMemcpyAsync(&a.npieces, a.poff.p + nv, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    sync();
    a.pv.ensure(a.npieces);
    { ++n_launch; k_piece_fill<<<grid(), THREADS, 0, s>>>(a.poff.p, nv, a.pv.p); }
    PCK(cudaGetLastError());
  }

  void build(uint32_t n, const uint64_t *r, const uint32_t *c, int mem) {
    nv = n;
    row.ensure((size_t)nv + 1);
    PCK(cudaMemcpyAsync(row.p, r, sizeof(uint64_t) * (nv + 1), kin(mem), s));
    PCK(cudaMemcpyAsync(&ne, row.p + nv, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    sync();
    if (ne >= (1ull << 31)) throw PprFail{SGS_ERR_INVALID, "more than 2^31-1 edges"};
    col.ensure(ne);
    if (ne) PCK(cudaMemcpyAsync(col.p, c, sizeof(uint32_t) * ne, kin(mem), s));
    err.ensure(1);
    PCK(cudaMemsetAsync(err.p, 0, sizeof(unsigned int), s));
    { ++n_launch; k_validate<<<grid(), THREADS, 0, s>>>(row.p, col.p, nv, ne, err.p); }
    unsigned int h = 0;
    PCK(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    sync();
    if (h & 2u) throw PprFail{SGS_ERR_INVALID, "row offsets must start at 0 and not decrease"};
    if (h & 1u) throw PprFail{SGS_ERR_INVALID, "column index out of range"};
    // CSC: sort (destination, CSR edge index) by destination (stable, so the
    // in-edges of a vertex keep CSR order), sources through the edge index.
    {
      Buf<uint32_t> src, dst_s, eid;
      src.ensure(ne);
      dst_s.ensure(ne);
      eid.ensure(ne);
      csrc.ensure(ne);
      ceid.ensure(ne);
      crow.ensure((size_t)nv + 1);
      { ++n_launch; k_edge_src<<<grid(), THREADS, 0, s>>>(row.p, nv, src.p); }
      { ++n_launch; k_iota<<<grid(), THREADS, 0, s>>>(eid.p, ne); }
      int bits = 1;
      while (bits < 32 && (1ull << bits) < nv) ++bits;
      size_t tb = 0;
      PCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, col.p, dst_s.p, eid.p, ceid.p, (int)ne, 0,
                                          bits, s));
      Buf<unsigned char> tmp;
      tmp.ensure(tb);
      PCK(cub::DeviceRadixSort::SortPairs(tmp.p, tb, col.p, dst_s.p, eid.p, ceid.p, (int)ne, 0,
                                          bits, s));
      { ++n_launch; k_csc_rows<<<grid(), THREADS, 0, s>>>(dst_s.p, ne, nv, crow.p); }
      { ++n_launch; k_gather_u32<<<grid(), THREADS, 0, s>>>(src.p, ceid.p, ne, csrc.p); }
      PCK(cudaGetLastError());
      sync();
    }
    pieces(in, crow.p, csrc.p);
    pieces(out, row.p, col.p);
    inv_s.ensure(nv);
    pr.ensure(ne);
    pc.ensure(ne);
    diff.ensure(64);
    sync();
  }

  // Loads a weight vector and forms inv_s, pr (CSR order) and pc (CSC order).
  void set_weights(const double *wt, int mem) {
    w.ensure(ne);
    if (ne) PCK(cudaMemcpyAsync(w.p, wt, sizeof(double) * ne, kin(mem), s));
    PCK(cudaMemsetAsync(err.p, 0, sizeof(unsigned int), s));
    { ++n_launch; k_row_probs<<<grid(), THREADS, 0, s>>>(row.p, nv, w.p, inv_s.p, pr.p, err.p); }
    { ++n_launch; k_csc_probs<<<grid(), THREADS, 0, s>>>(pr.p, ceid.p, ne, pc.p); }
    PCK(cudaGetLastError());
    unsigned int h = 0;
    PCK(cudaMemcpyAsync(&h, err.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    sync();
    if (h) throw PprFail{SGS_ERR_INVALID, "edge weights must be positive and finite"};
  }

  template <int LPE, int CPL>
  void launch_step(const Adj &a, const double *p, uint32_t K, double alpha, double c,
                   const double *B, const double *xin, double *xout, double *d) {
    { ++n_launch; k_ppr_step<LPE, CPL><<<rgrid((const void *)k_ppr_step<LPE, CPL>), THREADS, 0, s>>>(a.ptr, a.nbr, p, nv, a.pv.p, a.poff.p,
                                                    a.npieces, K, alpha, c, B, xin, xout, part.p, d); }
  }

  template <int L>
  void launch_grad(uint32_t K, double alpha, const double *Y, double *dst) {
    { ++n_launch; k_ppr_edge_grad<L><<<rgrid((const void *)k_ppr_edge_grad<L>), THREADS, 0, s>>>(row.p, col.p, inv_s.p, nv, out.pv.p, out.poff.p,
                                                  out.npieces, K, alpha, x.p, Y, g.p, dst); }
  }

  // One Jacobi step xin -> xout along `a` with probabilities p.
  void step(const Adj &a, const double *p, uint32_t K, double alpha, double c, const double *B,
            const double *xin, double *xout, double *d) {
    switch (K <= 32 ? lanes_per_edge(K) : 64) {
      case 1: launch_step<1, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      case 2: launch_step<2, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      case 4: launch_step<4, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      case 8: launch_step<8, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      case 16: launch_step<16, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      case 32: launch_step<32, 1>(a, p, K, alpha, c, B, xin, xout, d); break;
      default: launch_step<32, 2>(a, p, K, alpha, c, B, xin, xout, d); break;
    }
    if (a.npieces)
      { ++n_launch; k_ppr_finalize<<<rgrid((const void *)k_ppr_finalize), THREADS, 0, s>>>(a.pv.p, a.poff.p, a.npieces, K, alpha, c, B, xin,
                                                xout, part.p, d); }
  }

  // Jacobi steps (cur -> nxt, swap) until one step changes the state by
  // less than tol in L1; batches of 4, 8, ..., 32 steps between host reads
  // (the steps after the first converged one only move the state closer).
  template <class Step>
  int iterate(Step stepf, double *&cur, double *&nxt, double tol, uint32_t max_iter) {
    uint32_t it = 0, batch = 4;
    double hd[32];
    while (it < max_iter) {
      const uint32_t nb = std::min<uint32_t>(batch, max_iter - it);
      PCK(cudaMemsetAsync(diff.p, 0, sizeof(double) * nb, s));
      for (uint32_t b = 0; b < nb; ++b) {
        if (timing) PCK(cudaEventRecord(ev[2 * b], s));
        stepf(cur, nxt, diff.p + b);
        if (timing) PCK(cudaEventRecord(ev[2 * b + 1], s));
        std::swap(cur, nxt);
      }
      PCK(cudaGetLastError());
      PCK(cudaMemcpyAsync(hd, diff.p, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
      sync();
      if (timing)
        for (uint32_t b = 0; b < nb; ++b) {
          float ms = 0.f;
          PCK(cudaEventElapsedTime(&ms, ev[2 * b], ev[2 * b + 1]));
          st.steps_ms += ms;
        }
      it += nb;
      st.iters = (int32_t)it;
      for (uint32_t b = 0; b < nb; ++b)
        if (hd[b] < tol) return (int)it;
      batch = std::min<uint32_t>(batch * 2, 32);
    }
    return -1;
  }

  int forward(const double *T, uint32_t K, double alpha, double tol, uint32_t max_iter, double *X,
              int mem) {
    const uint64_t n = (uint64_t)nv * K;
    t.ensure(n);
    x.ensure(n);
    xn.ensure(n);
    part.ensure((uint64_t)std::max(in.npieces, out.npieces) * K);
    PCK(cudaMemcpyAsync(t.p, T, sizeof(double) * n, kin(mem), s));
    { ++n_launch; k_scale<<<grid(), THREADS, 0, s>>>(t.p, 1.0 - alpha, n, x.p); }
    double *cur = x.p, *nxt = xn.p;
    const int it = iterate(
        [&](double *a, double *b, double *d) { step(in, pc.p, K, alpha, 1.0 - alpha, t.p, a, b, d); },
        cur, nxt, tol, max_iter);
    PCK(cudaMemcpyAsync(X, cur, sizeof(double) * n, kout(mem), s));
    sync();
    return it;
  }

  int backward(const double *X, const double *G, uint32_t K, double alpha, double tol,
               uint32_t max_iter, double *gw, double *gT, int mem) {
    const uint64_t n = (uint64_t)nv * K;
    x.ensure(n);
    g.ensure(n);
    y.ensure(n);
    yn.ensure(n);
    part.ensure((uint64_t)std::max(in.npieces, out.npieces) * K);
    PCK(cudaMemcpyAsync(x.p, X, sizeof(double) * n, kin(mem), s));
    PCK(cudaMemcpyAsync(g.p, G, sizeof(double) * n, kin(mem), s));
    PCK(cudaMemcpyAsync(y.p, g.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    double *cur = y.p, *nxt = yn.p;
    const int it = iterate(
        [&](double *a, double *b, double *d) { step(out, pr.p, K, alpha, 1.0, g.p, a, b, d); },
        cur, nxt, tol, max_iter);
    if (it < 0) return it;
    if (gw && ne) {
      Buf<double> tmp;
      double *dst = gw;
      if (mem == SGS_MEM_HOST) {
        tmp.ensure(ne);
        dst = tmp.p;
      }
      switch (lanes_per_edge(K)) {
        case 1: launch_grad<1>(K, alpha, cur, dst); break;
        case 2: launch_grad<2>(K, alpha, cur, dst); break;
        case 4: launch_grad<4>(K, alpha, cur, dst); break;
        case 8: launch_grad<8>(K, alpha, cur, dst); break;
        case 16: launch_grad<16>(K, alpha, cur, dst); break;
        default: launch_grad<32>(K, alpha, cur, dst); break;
      }
      PCK(cudaGetLastError());
      if (mem == SGS_MEM_HOST) PCK(cudaMemcpyAsync(gw, dst, sizeof(double) * ne, kout(mem), s));
      sync();
    }
    if (gT) {
      Buf<double> tmp;
      double *dst = gT;
      if (mem == SGS_MEM_HOST) {
        tmp.ensure(n);
        dst = tmp.p;
      }
      { ++n_launch; k_scale<<<grid(), THREADS, 0, s>>>(cur, 1.0 - alpha, n, dst); }
      PCK(cudaGetLastError());
      if (mem == SGS_MEM_HOST) PCK(cudaMemcpyAsync(gT, dst, sizeof(double) * n, kout(mem), s));
      sync();
    }
    sync();
    return it;
  }
};

template <class F>
static int pguard(F &&f) {
  try {
    f();
    return SGS_OK;
  } catch (const PprFail &e) {
    sgs::set_last_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc &) {
    sgs::set_last_error("host allocation failed");
    return SGS_ERR_OOM;
  }
}

static bool bad_args(double alpha, uint32_t K) {
  if (!(alpha > 0.0 && alpha < 1.0)) {
    sgs::set_last_error("alpha must be in (0, 1)");
    return true;
  }
  if (K == 0) {
    sgs::set_last_error("K must be at least 1");
    return true;
  }
  return false;
}

extern "C" {

SGS_API int sgs_ppr_create_csr(int device, uint32_t nv, const uint64_t *row, const uint32_t *col,
                               int mem, sgs_ppr **out) {
  if (!out || !row || !col) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  *out = nullptr;
  if (nv == 0) {
    sgs::set_last_error("empty graph");
    return SGS_ERR_INVALID;
  }
  return pguard([&] {
    auto p = std::make_unique<sgs_ppr>();
    p->dev = device;
    PCK(cudaSetDevice(device));
    PCK(cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, device));
    PCK(cudaStreamCreateWithFlags(&p->s, cudaStreamNonBlocking));
    p->build(nv, row, col, mem);
    *out = p.release();
  });
}

SGS_API int sgs_ppr_create(sgs_engine *e, sgs_ppr **out) {
  if (!e || !out) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  sgs_engine_stats st;
  int rc = sgs_get_engine_stats(e, &st);
  if (rc) return rc;
  std::vector<uint64_t> row((size_t)st.nv + 1);
  std::vector<uint32_t> col(std::max<uint64_t>(st.ne, 1));
  // the export leaves the engine's device current
  rc = sgs_graph_export(e, row.data(), col.data(), nullptr, SGS_MEM_HOST);
  if (rc) return rc;
  int dev = 0;
  cudaGetDevice(&dev);
  return sgs_ppr_create_csr(dev, (uint32_t)st.nv, row.data(), col.data(), SGS_MEM_HOST, out);
}

SGS_API int sgs_ppr_destroy(sgs_ppr *p) {
  if (p) {
    cudaSetDevice(p->dev);
    cudaStreamSynchronize(p->s);
    delete p;
  }
  return SGS_OK;
}

SGS_API int sgs_ppr_info(sgs_ppr *p, uint32_t *nv, uint64_t *ne) {
  if (!p || !nv || !ne) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  *nv = p->nv;
  *ne = p->ne;
  return SGS_OK;
}

SGS_API int sgs_ppr_timing(sgs_ppr *p, int enable) {
  if (!p) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  p->timing = enable != 0;
  return SGS_OK;
}

SGS_API int sgs_ppr_get_stats(sgs_ppr *p, sgs_ppr_stats *out) {
  if (!p || !out) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  p->st.pieces_in = p->in.npieces;
  p->st.pieces_out = p->out.npieces;
  p->st.kernel_launches = p->n_launch;
  *out = p->st;
  return SGS_OK;
}

SGS_API int sgs_ppr_export(sgs_ppr *p, uint64_t *row, uint32_t *col, int mem) {
  if (!p || !row || !col) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  return pguard([&] {
    PCK(cudaSetDevice(p->dev));
    PCK(cudaMemcpyAsync(row, p->row.p, sizeof(uint64_t) * (p->nv + 1), p->kout(mem), p->s));
    if (p->ne) PCK(cudaMemcpyAsync(col, p->col.p, sizeof(uint32_t) * p->ne, p->kout(mem), p->s));
    p->sync();
  });
}

SGS_API int sgs_ppr_forward(sgs_ppr *p, const double *w, const double *T, uint32_t K, double alpha,
                            double tol, uint32_t max_iter, double *X, int *iters, int mem) {
  if (!p || !w || !T || !X) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  if (bad_args(alpha, K)) return SGS_ERR_INVALID;
  return pguard([&] {
    PCK(cudaSetDevice(p->dev));
    p->set_weights(w, mem);
    p->call_begin();
    p->st.bytes_alg_step = p->step_bytes(K);
    const int it = p->forward(T, K, alpha, tol, max_iter, X, mem);
    p->call_end();
    if (iters) *iters = it;
    if (it < 0) throw PprFail{SGS_ERR_NOCONV, "PPR forward did not converge"};
  });
}

SGS_API int sgs_ppr_backward(sgs_ppr *p, const double *w, const double *X, const double *G,
                             uint32_t K, double alpha, double tol, uint32_t max_iter, double *gw,
                             double *gT, int *iters, int mem) {
  if (!p || !w || !X || !G) {
    sgs::set_last_error("null argument");
    return SGS_ERR_INVALID;
  }
  if (bad_args(alpha, K)) return SGS_ERR_INVALID;
  return pguard([&] {
    PCK(cudaSetDevice(p->dev));
    p->set_weights(w, mem);
    p->call_begin();
    p->st.bytes_alg_step = p->step_bytes(K);
    const int it = p->backward(X, G, K, alpha, tol, max_iter, gw, gT, mem);
    p->call_end();
    if (iters) *iters = it;
    if (it < 0) throw PprFail{SGS_ERR_NOCONV, "PPR adjoint did not converge"};
  });
}

}  // extern "C"
