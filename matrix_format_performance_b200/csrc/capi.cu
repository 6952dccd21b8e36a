// C ABI: plans, kernel launches, device-resident matrix handles and timing.
#include "host_common.h"
#include "spmv_kernels.cuh"
#include "spmv_stream.cuh"
#include "spmv_lowp.cuh"
#include "mlp.cuh"
#include "spmv_probe.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

using namespace mfp;
namespace d = mfp::dev;

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  return fail(MFP_ERROR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define CUDA_TRY(expr, what)                    \
  do {                                          \
    cudaError_t _e = (expr);                    \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

// COO, the hybrid's tail and row-ordered SCOO keep their rows in handles as
// 16-bit offsets where they fit (1), or always as 32-bit ids (0); COO and the
// hybrid's tail as 8-bit offsets where every tile allows them (ROWS8 1).
#ifndef MFP_COMPACT_ROWS
#define MFP_COMPACT_ROWS 1
#endif
#ifndef MFP_COMPACT_ROWS8
#define MFP_COMPACT_ROWS8 1
#endif
inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline bool aligned32(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; }
// Per-lane group loads of the warp-tile kernels: 2 = one 32-byte load per
// array, 1 = two 16-byte loads, 0 = element by element.
inline int vec_level(const void *a, const void *b, const void *c = nullptr) {
  if (aligned32(a) && aligned32(b) && (!c || aligned32(c))) return 2;
  return aligned16(a) && aligned16(b) && (!c || aligned16(c)) ? 1 : 0;
}
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline uint32_t ceil_div(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

int check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, what);
  return ok();
}

// Per (kernel, device): the dynamic shared-memory limit set so far and the
// resident CTAs per SM of a persistent launch.
struct kernel_cache {
  std::mutex mu;
  std::map<std::pair<const void *, int>, size_t> limit;
  std::map<std::pair<const void *, int>, int> occupancy;
  std::map<int, int> sms;
};
kernel_cache &kcache() {
  static kernel_cache c;
  return c;
}

// Raises `k`'s dynamic shared-memory limit on the current device to `dyn`.
int ensure_dyn_smem(const void *k, size_t dyn, const char *name) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  auto &c = kcache();
  std::lock_guard<std::mutex> g(c.mu);
  size_t &lim = c.limit[{k, dev}];
  if (dyn <= lim) return ok();
  const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(MFP_ERROR_CUDA, "cudaFuncSetAttribute(%s, %zu dynamic bytes): %s", name, dyn, cudaGetErrorString(e));
  }
  lim = dyn;
  return ok();
}

// Resident CTAs per SM of `k` (block `threads`, `dyn` dynamic bytes) times the
// SM count of the current device: the grid of a persistent launch.
int persistent_grid(const void *k, int threads, size_t dyn, uint32_t *grid) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  auto &c = kcache();
  std::lock_guard<std::mutex> g(c.mu);
  auto it = c.occupancy.find({k, dev});
  if (it == c.occupancy.end()) {
    int blocks = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, threads, dyn),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    it = c.occupancy.emplace(std::make_pair(k, dev), std::max(1, blocks)).first;
  }
  auto sit = c.sms.find(dev);
  if (sit == c.sms.end()) {
    int n = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    sit = c.sms.emplace(dev, n).first;
  }
  *grid = (uint32_t)it->second * (uint32_t)sit->second;
  return ok();
}

template <typename T>
int dmalloc(T **p, size_t count, size_t *acct = nullptr) {
  *p = nullptr;
  if (count == 0) return MFP_SUCCESS;
  const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? MFP_ERROR_OUT_OF_MEMORY : MFP_ERROR_CUDA,
                "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
  }
  if (acct) *acct += count * sizeof(T);
  return MFP_SUCCESS;
}
template <typename T>
int upload(T **p, const T *host, size_t count, size_t *acct = nullptr) {
  int st = dmalloc(p, count, acct);
  if (st) return st;
  if (count) CUDA_TRY(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  return MFP_SUCCESS;
}

}  // namespace

// ---------------------------------------------------------------------------
// CSR plan
// ---------------------------------------------------------------------------
namespace {
// Streaming CSR kernel variants: chunk of CH elements, S pipeline stages.
// Variant 0 (config.kernel = 2): 2048-element chunks; variant 1 (= 3):
// 1024-element chunks with a deeper ring.
template <typename T, int V>
struct stream_cfg;
template <>
struct stream_cfg<float, 0> {
  static constexpr int CH = 2048, S = 3;
};
template <>
struct stream_cfg<double, 0> {
  static constexpr int CH = 2048, S = 2;
};
template <>
struct stream_cfg<float, 1> {
  static constexpr int CH = 1024, S = 4;
};
template <>
struct stream_cfg<double, 1> {
  static constexpr int CH = 1024, S = 3;
};
template <typename T, int V>
constexpr size_t stream_smem_bytes() {
  using C = stream_cfg<T, V>;
  return sizeof(d::stream_smem<T, C::CH, C::S>) + d::kCrowCap * sizeof(uint32_t);
}
struct stream_plan {
  uint32_t chunk = 0, nchunks = 0;
  uint32_t *chunk_row = nullptr;
  uint32_t grid = 0, chunks_per_cta = 0, n_contrib = 0, slots = 0;
  d::stream_edge *edges = nullptr;
  d::long_piece *contrib = nullptr;
  double *partials = nullptr;
  uint32_t *counters = nullptr;
};
}  // namespace

struct mfp_csr_plan {
  uint32_t *error = nullptr;
  stream_plan sp[2];  // per value type (f32, f64): chunking and grid depend on both
  int device = 0;
  int algo = 0;
  mfp_csr_config cfg{};
  uint32_t assist_thr = 64;
  uint32_t rows = 0, cols = 0, nnz = 0;
  uint32_t n_main = 0, n_pieces = 0, n_long = 0;
  d::long_piece *pieces = nullptr;
  double *partials = nullptr;
  uint32_t *counters = nullptr;
  uint32_t *row_blocks = nullptr;
  uint32_t *order = nullptr;  // work items heaviest first (n_main + n_pieces)
  // warp-tile kernel (CSR vector on short rows): the row of the element before
  // each 256-element tile, and the COO-style workspace of the fix-up pass
  uint4 *blk = nullptr;  // per row block: element range and flags (see csr_args::blk)
  bool fast = false;     // row blocks without long rows start their loads before the row_ptr barrier
  bool binned = false;   // CSR scalar on the CSR-Adaptive bins, one thread per row
  bool tile = false;
  uint32_t *tile_prev = nullptr;
  void *tile_ws = nullptr;
  size_t tile_ws_bytes = 0;
  size_t device_bytes = 0;
};

// Launch the CSR family's work items heaviest first (1) or in index order (0).
#ifndef MFP_CSR_ORDER
#define MFP_CSR_ORDER 1
#endif

namespace {
// COO workspace: a 16-byte header (the first and last row holding elements;
// its error word stays 0: the two-pass COO has no waits) and, per 256-element
// warp tile, the head and tail partial sums (8 bytes each, FP64-sized), the
// flags and the tail row.  Every call rewrites what it reads: no
// initialisation.
size_t coo_ws_bytes(uint32_t nnz) {
  const uint64_t wt = (nnz + (uint64_t)d::kWarpTile - 1) / d::kWarpTile;
  return sizeof(d::coo_ws_header) + wt * 24u;
}
constexpr uint32_t kDefaultLong = 4096;
constexpr uint32_t kDefaultAssist = 64;
// One CTA per long row up to 65,536 elements: on the power-law matrix (rows
// up to 50,000) pieces of 4,096 / 16,384 / 65,536 elements took CSR scalar
// to 0.191 / 0.188 / 0.184 ms and CSR-Adaptive to 0.172 / 0.168 / 0.164 ms
// (each extra piece adds a CTA-wide FP64 reduction and the combine).
constexpr uint32_t kDefaultPiece = 65536;
constexpr uint32_t kFp64Rows = 4096;  // rows longer than this accumulate in FP64
constexpr uint32_t kMaxBin = d::kChunk - 4;
}  // namespace

namespace {
template <typename T, int V, int MODE>
int stream_occupancy() {
  using C = stream_cfg<T, V>;
  auto k = d::csr_stream_kernel<T, MODE, C::CH, C::S>;
  const int smem = (int)stream_smem_bytes<T, V>();
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) cudaGetLastError();
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, d::kBlock, smem) != cudaSuccess) {
    cudaGetLastError();
    blocks = 2;
  }
  return std::max(1, blocks);
}
template <typename T, int V>
int stream_occupancy_algo(int algo) {
  return algo == 0 ? stream_occupancy<T, V, 0>() : algo == 1 ? stream_occupancy<T, V, 1>() : stream_occupancy<T, V, 2>();
}

// Fixed chunks of `chunk` elements, statically partitioned over `target`
// persistent CTAs, and the contributions of the rows split between two CTA
// ranges (an ordered partial-sum slot per CTA the row touches).
int build_stream_plan(stream_plan &sp, uint32_t rows, uint32_t nnz, const uint32_t *rp, uint32_t chunk,
                      uint32_t target, size_t *acct) {
  sp.chunk = chunk;
  sp.nchunks = ceil_div(nnz, chunk);
  if (sp.nchunks == 0) return MFP_SUCCESS;
  std::vector<uint32_t> cr((size_t)sp.nchunks + 1);
  for (uint32_t k = 0; k < sp.nchunks; ++k)
    cr[k] = (uint32_t)(std::lower_bound(rp, rp + rows + 1, k * chunk) - rp);
  cr[sp.nchunks] = rows;
  const uint32_t K = ceil_div(sp.nchunks, std::max(1u, target));
  sp.chunks_per_cta = K;
  sp.grid = ceil_div(sp.nchunks, K);
  const uint64_t span = (uint64_t)K * chunk;  // elements per CTA
  std::vector<d::stream_edge> edges(sp.grid, d::stream_edge{d::kNoPiece, d::kNoPiece});
  std::vector<d::long_piece> contrib;
  uint32_t slots = 0, counter = 0;
  uint32_t last_row = UINT32_MAX;
  for (uint32_t c = 0; c + 1 < sp.grid; ++c) {
    const uint64_t C1 = std::min<uint64_t>((uint64_t)(c + 1) * span, nnz);
    // the row holding element C1 - 1, if it continues past C1
    const uint32_t r = (uint32_t)(std::upper_bound(rp, rp + rows + 1, (uint32_t)(C1 - 1)) - rp) - 1;
    if (rp[r + 1] <= C1 || r == last_row) continue;
    last_row = r;
    const uint32_t cs = (uint32_t)(rp[r] / span), ce = (uint32_t)((rp[r + 1] - 1) / span);
    const uint32_t np = ce - cs + 1;
    for (uint32_t q = cs; q <= ce; ++q) {
      d::long_piece pc{};
      pc.row = r;
      pc.slot_base = slots;
      pc.piece = q - cs;
      pc.npieces = np;
      pc.counter = counter;
      pc.fp64 = (rp[r + 1] - rp[r]) > kFp64Rows;
      const uint32_t idx = (uint32_t)contrib.size();
      contrib.push_back(pc);
      if (q != cs) edges[q].head = idx;
      if (q != ce) edges[q].tail = idx;
    }
    slots += np;
    ++counter;
  }
  sp.n_contrib = (uint32_t)contrib.size();
  sp.slots = slots;
  int st;
  if ((st = upload(&sp.chunk_row, cr.data(), cr.size(), acct)) ||
      (st = upload(&sp.edges, edges.data(), edges.size(), acct)) ||
      (st = upload(&sp.contrib, contrib.data(), contrib.size(), acct)) ||
      (st = dmalloc(&sp.partials, slots, acct)) || (st = dmalloc(&sp.counters, counter, acct)))
    return st;
  if (counter) CUDA_TRY(cudaMemset(sp.counters, 0, counter * sizeof(uint32_t)), "cudaMemset counters");
  return MFP_SUCCESS;
}

void free_stream_plan(stream_plan &sp) {
  cudaFree(sp.chunk_row);
  cudaFree(sp.edges);
  cudaFree(sp.contrib);
  cudaFree(sp.partials);
  cudaFree(sp.counters);
  sp = stream_plan{};
}
}  // namespace

// Streaming-kernel plans for both value types; variant from config.kernel.
int build_stream_plans(mfp_csr_plan *plan, const uint32_t *rp) {
  if (plan->nnz == 0 || (plan->cfg.kernel != 2 && plan->cfg.kernel != 3)) return MFP_SUCCESS;
  int st;
  if ((st = dmalloc(&plan->error, 1, &plan->device_bytes))) return st;
  CUDA_TRY(cudaMemset(plan->error, 0, sizeof(uint32_t)), "cudaMemset error word");
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan->device);
  const bool v1 = plan->cfg.kernel == 3;
  const int occ32 = v1 ? stream_occupancy_algo<float, 1>(plan->algo) : stream_occupancy_algo<float, 0>(plan->algo);
  const int occ64 = v1 ? stream_occupancy_algo<double, 1>(plan->algo) : stream_occupancy_algo<double, 0>(plan->algo);
  const uint32_t ch32 = v1 ? stream_cfg<float, 1>::CH : stream_cfg<float, 0>::CH;
  const uint32_t ch64 = v1 ? stream_cfg<double, 1>::CH : stream_cfg<double, 0>::CH;
  if ((st = build_stream_plan(plan->sp[0], plan->rows, plan->nnz, rp, ch32, (uint32_t)(sms * occ32),
                              &plan->device_bytes)) ||
      (st = build_stream_plan(plan->sp[1], plan->rows, plan->nnz, rp, ch64, (uint32_t)(sms * occ64),
                              &plan->device_bytes)))
    return st;
  return MFP_SUCCESS;
}

extern "C" int mfp_csr_plan_create(uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp,
                                   int algo, const mfp_csr_config *config, mfp_csr_plan **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "plan output is NULL");
  *out = nullptr;
  if (algo < 0 || algo > 2) return fail(MFP_ERROR_INVALID_VALUE, "unknown CSR algorithm %d", algo);
  int st = check_row_ptr(rows, nnz, rp);
  if (st) return st;
  mfp_csr_config cfg = config ? *config : mfp_csr_config{};
  auto *plan = new mfp_csr_plan();
  cudaGetDevice(&plan->device);
  plan->algo = algo;
  plan->rows = rows;
  plan->cols = cols;
  plan->nnz = nnz;
  if (cfg.piece_nnz == 0) cfg.piece_nnz = kDefaultPiece;
  cfg.piece_nnz = std::max(cfg.piece_nnz, 256u);
  // CSR scalar on short rows (mean length below 16, automatic kernel, not
  // the exact-order setting): the CSR-Adaptive bins, which balance elements
  // per CTA, with each row summed by one thread in CSR order.  Measured on
  // B200 against 256-row blocks, FP32: power-law 4M 0.185 -> 0.162 ms,
  // 4M rows of 6-9 uniform elements 0.166 -> 0.160 ms.  From mean 16 (the
  // 27-point stencil, banded 8M) a bin holds too few rows for its threads.
  const bool exact = cfg.long_row_threshold == UINT32_MAX && cfg.assist_threshold == UINT32_MAX;
  plan->binned = algo == MFP_CSR_SCALAR && cfg.kernel == 0 && !exact && rows && (double)nnz / rows < 16.0;
  if (algo == MFP_CSR_ADAPTIVE || plan->binned)
    cfg.bin_nnz = cfg.bin_nnz ? std::min(cfg.bin_nnz, kMaxBin) : kMaxBin;
  if (algo == MFP_CSR_ADAPTIVE) {
    // rows longer than a bin and up to 4096 elements: one CTA each (plain
    // float), longer ones in FP64 pieces
    if (cfg.long_row_threshold == 0) cfg.long_row_threshold = std::max(cfg.bin_nnz, kDefaultLong);
  } else {
    if (cfg.long_row_threshold == 0) cfg.long_row_threshold = kDefaultLong;
  }
  if (algo == MFP_CSR_VECTOR) {
    uint32_t L = cfg.vector_lanes;
    // auto below a mean row length of 64: the warp-tile kernel, where lanes
    // share rows through the segmented scan.  Measured on B200 against 2 and 4
    // lanes per row: power-law 4M 0.187 ms (2 lanes 0.240), 27-point stencil
    // 0.153 ms (0.178), banded 8M 0.599 ms (0.669), FP32.
    plan->tile = L == 0 && cfg.kernel == 0 && rows && (double)nnz / rows < 64.0;
    if (L == 0) {
      // Measured on B200 over 2,200 seeded matrices (uniform, Zipf, banded,
      // block-diagonal, stencil, dense-row families) and the 4M-row power-law
      // matrix: with products staged in shared memory a narrow group (more
      // rows in flight, longer lane-strided sums) wins; 4 lanes was the best
      // of {4, 8, 32, prevpow2(mean)} at every mean length >= 3, and 2 lanes
      // beat 4 on the power-law matrix (mean 7.5).
      const double mean = rows ? (double)nnz / rows : 1.0;
      L = mean < 12.0 ? 2u : 4u;
    }
    if (L < 2 || L > 32 || (L & (L - 1))) {
      delete plan;
      return fail(MFP_ERROR_INVALID_VALUE, "vector_lanes must be a power of two in [2, 32]");
    }
    cfg.vector_lanes = L;
  }
  if (cfg.kernel == 4) plan->tile = true;  // the warp-tile kernel on request, any algorithm
  if (nnz == 0) plan->tile = false;
  plan->assist_thr = cfg.assist_threshold ? cfg.assist_threshold : kDefaultAssist;
  plan->cfg = cfg;

  // long rows -> pieces of at most piece_nnz elements
  std::vector<d::long_piece> pieces;
  uint32_t slots = 0, nlong = 0;
  for (uint32_t r = 0; r < rows; ++r) {
    const uint32_t len = rp[r + 1] - rp[r];
    if (len <= cfg.long_row_threshold) continue;
    const uint32_t np = ceil_div(len, cfg.piece_nnz);
    for (uint32_t k = 0; k < np; ++k) {
      d::long_piece pc{};
      pc.row = r;
      pc.e0 = rp[r] + k * cfg.piece_nnz;
      pc.e1 = std::min(rp[r + 1], pc.e0 + cfg.piece_nnz);
      pc.slot_base = slots;
      pc.piece = k;
      pc.npieces = np;
      pc.counter = nlong;
      pc.fp64 = len > kFp64Rows ? 1u : 0u;
      pieces.push_back(pc);
    }
    if (np > 1) slots += np;
    ++nlong;
  }
  std::vector<uint32_t> blocks;
  if (algo == MFP_CSR_ADAPTIVE || plan->binned) {
    blocks.push_back(0);
    uint32_t cur_rows = 0, cur_nnz = 0;
    const uint32_t max_rows = 4 * d::kBlock;
    for (uint32_t r = 0; r < rows; ++r) {
      const uint32_t len = rp[r + 1] - rp[r];
      const bool own = len > cfg.long_row_threshold || len > cfg.bin_nnz;
      if (cur_rows && (own || cur_nnz + len > cfg.bin_nnz || cur_rows >= max_rows)) {
        blocks.push_back(r);
        cur_rows = cur_nnz = 0;
      }
      if (own) {
        blocks.push_back(r + 1);
        continue;
      }
      cur_rows++;
      cur_nnz += len;
    }
    if (cur_rows) blocks.push_back(rows);
    plan->n_main = (uint32_t)blocks.size() - 1;
  } else if (algo == MFP_CSR_SCALAR) {
    plan->n_main = ceil_div(rows, d::kBlock);
  } else {
    plan->n_main = ceil_div(rows, d::kBlock);
  }
  plan->n_pieces = (uint32_t)pieces.size();
  plan->n_long = nlong;
  if ((st = build_stream_plans(plan, rp))) {
    mfp_csr_plan_destroy(plan);
    return st;
  }
  if ((uint64_t)plan->n_main + plan->n_pieces > 0x7fffffffull) {
    delete plan;
    return fail(MFP_ERROR_TOO_LARGE, "grid too large");
  }
  // launch order: work items by element count, heaviest first (stable)
  std::vector<uint32_t> order((size_t)plan->n_main + plan->n_pieces);
  {
    std::vector<uint64_t> cost(order.size());
    for (uint32_t b = 0; b < plan->n_main; ++b) {
      const bool bins = algo == MFP_CSR_ADAPTIVE || plan->binned;
      const uint32_t r0 = bins ? blocks[b] : b * d::kBlock;
      const uint32_t r1 = bins ? blocks[b + 1] : std::min(rows, r0 + d::kBlock);
      uint64_t c = r1 - r0;
      for (uint32_t r = r0; r < r1; ++r) {
        const uint32_t len = rp[r + 1] - rp[r];
        if (len <= cfg.long_row_threshold) c += len;
      }
      cost[b] = c;
    }
    for (uint32_t k = 0; k < plan->n_pieces; ++k) cost[plan->n_main + k] = pieces[k].e1 - pieces[k].e0;
    for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  }
  if ((st = upload(&plan->order, order.data(), order.size(), &plan->device_bytes)) ||
      (st = upload(&plan->pieces, pieces.data(), pieces.size(), &plan->device_bytes)) ||
      (st = dmalloc(&plan->partials, slots, &plan->device_bytes)) ||
      (st = dmalloc(&plan->counters, nlong, &plan->device_bytes)) ||
      (st = upload(&plan->row_blocks, blocks.data(), blocks.size(), &plan->device_bytes))) {
    mfp_csr_plan_destroy(plan);
    return st;
  }
  // row blocks that start their loads before the row_ptr barrier: measured
  // faster for lanes per row and for long rows (mean length 16 and up)
  plan->fast = algo != MFP_CSR_ADAPTIVE && (algo == MFP_CSR_VECTOR || (rows && (double)nnz / rows >= 16.0));
  if (plan->fast) {
    // per row block: its element range and whether it holds a long or an
    // assisted row
    std::vector<uint4> br(plan->n_main);
    for (uint32_t b = 0; b < plan->n_main; ++b) {
      const uint32_t r0 = b * d::kBlock;
      const uint32_t r1 = std::min(rows, r0 + d::kBlock);
      uint32_t flags = 0;
      for (uint32_t r = r0; r < r1; ++r) {
        const uint32_t len = rp[r + 1] - rp[r];
        if (len > cfg.long_row_threshold) flags |= 1u;
        else if (len > plan->assist_thr) flags |= 2u;
      }
      br[b] = make_uint4(rp[r0], rp[r1], flags, 0u);
    }
    if ((st = upload(&plan->blk, br.data(), br.size(), &plan->device_bytes))) {
      mfp_csr_plan_destroy(plan);
      return st;
    }
  }
  if (plan->tile) {
    // the row holding element 256 w - 1, for every warp tile w > 0
    const uint32_t n_wt = ceil_div(nnz, d::kWarpTile);
    std::vector<uint32_t> prev(n_wt);
    prev[0] = d::kNoRow;
    for (uint32_t w = 1; w < n_wt; ++w) {
      const uint32_t e = w * d::kWarpTile - 1u;
      prev[w] = (uint32_t)(std::upper_bound(rp, rp + rows + 1, e) - rp) - 1u;
    }
    plan->tile_ws_bytes = coo_ws_bytes(nnz);
    unsigned char *ws = nullptr;
    if ((st = upload(&plan->tile_prev, prev.data(), prev.size(), &plan->device_bytes)) ||
        (st = dmalloc(&ws, plan->tile_ws_bytes, &plan->device_bytes))) {
      mfp_csr_plan_destroy(plan);
      return st;
    }
    plan->tile_ws = ws;
  }
  if (nlong) {
    const cudaError_t e = cudaMemset(plan->counters, 0, nlong * sizeof(uint32_t));
    if (e != cudaSuccess) {
      mfp_csr_plan_destroy(plan);
      return cuda_fail(e, "cudaMemset counters");
    }
  }
  *out = plan;
  return ok();
}

extern "C" int mfp_csr_plan_destroy(mfp_csr_plan *plan) {
  if (!plan) return ok();
  cudaFree(plan->pieces);
  cudaFree(plan->partials);
  cudaFree(plan->counters);
  cudaFree(plan->row_blocks);
  cudaFree(plan->order);
  cudaFree(plan->error);
  cudaFree(plan->tile_prev);
  cudaFree(plan->tile_ws);
  cudaFree(plan->blk);
  free_stream_plan(plan->sp[0]);
  free_stream_plan(plan->sp[1]);
  delete plan;
  return ok();
}

extern "C" int mfp_csr_plan_get_config(const mfp_csr_plan *plan, int *algo, mfp_csr_config *cfg,
                                       uint32_t *long_rows, uint32_t *pieces) {
  if (!plan) return fail(MFP_ERROR_INVALID_VALUE, "plan is NULL");
  if (algo) *algo = plan->algo;
  if (cfg) {
    *cfg = plan->cfg;
    cfg->assist_threshold = plan->assist_thr;
  }
  if (long_rows) *long_rows = plan->n_long;
  if (pieces) *pieces = plan->n_pieces;
  return ok();
}

namespace {
template <typename T>
int fill(uint64_t n, T *v, T value, void *stream);

template <typename T, int V>
void launch_stream(int algo, uint32_t grid, cudaStream_t s, const d::stream_args<T> &S) {
  using C = stream_cfg<T, V>;
  const size_t smem = stream_smem_bytes<T, V>();
  switch (algo) {
    case 0: d::csr_stream_kernel<T, 0, C::CH, C::S><<<grid, d::kBlock, smem, s>>>(S); break;
    case 1: d::csr_stream_kernel<T, 1, C::CH, C::S><<<grid, d::kBlock, smem, s>>>(S); break;
    default: d::csr_stream_kernel<T, 2, C::CH, C::S><<<grid, d::kBlock, smem, s>>>(S); break;
  }
}

template <typename T>
int csr_tile_spmv(const mfp_csr_plan *plan, const T *data, const uint32_t *cols, const uint32_t *rp, const T *x,
                  T *y, cudaStream_t s);

template <typename T>
int csr_spmv(const mfp_csr_plan *plan, const T *data, const uint32_t *cols, const uint32_t *rp, const T *x,
             T *y, void *stream) {
  if (!plan) return fail(MFP_ERROR_INVALID_VALUE, "plan is NULL");
  if (plan->rows == 0) return ok();
  if (!rp || !y || (plan->nnz && (!data || !cols || !x))) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  d::csr_args<T> A{};
  A.n_rows = plan->rows;
  A.row_ptr = rp;
  A.cols = cols;
  A.vals = data;
  A.x = x;
  A.y = y;
  A.long_thr = plan->cfg.long_row_threshold;
  A.assist_thr = plan->assist_thr;
  A.lanes = plan->cfg.vector_lanes ? plan->cfg.vector_lanes : 32;
  A.row_blocks = plan->row_blocks;
  A.n_main = plan->n_main;
  A.n_pieces = plan->n_pieces;
  A.pieces = plan->pieces;
  A.partials = plan->partials;
  A.counters = plan->counters;
  A.order = MFP_CSR_ORDER ? plan->order : nullptr;
  A.blk = plan->blk;
  const bool vec = aligned16(data) && aligned16(cols);
  cudaStream_t s = as_stream(stream);
  if (plan->nnz == 0) return fill<T>(plan->rows, y, T(0), stream);
  const stream_plan &sp = plan->sp[sizeof(T) == 8 ? 1 : 0];
  // the exact-order configuration keeps every row in one thread's sequential
  // sum, which only the row-block kernel does for rows split between CTAs
  const bool exact_order = plan->cfg.long_row_threshold == UINT32_MAX && plan->assist_thr == UINT32_MAX;
  if (vec && aligned16(rp) && sp.grid && !exact_order && (plan->cfg.kernel == 2 || plan->cfg.kernel == 3)) {
    d::stream_args<T> S{};
    S.n_rows = plan->rows;
    S.nnz = plan->nnz;
    S.nchunks = sp.nchunks;
    S.chunks_per_cta = sp.chunks_per_cta;
    S.row_ptr = rp;
    S.cols = cols;
    S.vals = data;
    S.x = x;
    S.y = y;
    S.chunk_row = sp.chunk_row;
    S.edges = sp.edges;
    S.contrib = sp.contrib;
    S.partials = sp.partials;
    S.counters = sp.counters;
    S.error = plan->error;
    S.assist_thr = plan->assist_thr;
    S.lanes = A.lanes;
    S.fp64_thr = kFp64Rows;
    if (plan->cfg.kernel == 3)
      launch_stream<T, 1>(plan->algo, sp.grid, s, S);
    else
      launch_stream<T, 0>(plan->algo, sp.grid, s, S);
    return check_launch("csr_stream_kernel launch");
  }
  if (plan->tile && !exact_order) return csr_tile_spmv<T>(plan, data, cols, rp, x, y, s);
  const uint32_t grid = plan->n_main + plan->n_pieces;
  if (grid == 0) return ok();
#define MFP_CSR_LAUNCH(ALGO, FAST)                                                   \
  if (vec)                                                                           \
    d::csr_kernel<T, ALGO, true, FAST><<<grid, d::kBlock, 0, s>>>(A);                \
  else                                                                               \
    d::csr_kernel<T, ALGO, false, FAST><<<grid, d::kBlock, 0, s>>>(A);
  const bool fast = plan->fast && plan->blk;
  switch (plan->algo) {
    case 0:
      if (plan->binned) {
        MFP_CSR_LAUNCH(3, false)
      } else if (fast) {
        MFP_CSR_LAUNCH(0, true)
      } else {
        MFP_CSR_LAUNCH(0, false)
      }
      break;
    case 1:
      if (fast) { MFP_CSR_LAUNCH(1, true) } else { MFP_CSR_LAUNCH(1, false) }
      break;
    default: MFP_CSR_LAUNCH(2, false) break;
  }
#undef MFP_CSR_LAUNCH
  return check_launch("csr_kernel launch");
}

template <typename T>
int ell_spmv(uint32_t rows, uint32_t width, const T *data, const uint32_t *cols, const T *x, T *y,
             void *stream) {
  if (rows == 0) return ok();
  if (!y || (width && (!data || !cols || !x))) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  const bool vec = (rows % 4 == 0) && aligned16(data) && aligned16(cols) && aligned16(y);
  cudaStream_t s = as_stream(stream);
  if (vec)
    d::ell_kernel<T, true><<<ceil_div(rows / 4, d::kBlock), d::kBlock, 0, s>>>(rows, width, data, cols, x, y);
  else
    d::ell_kernel<T, false><<<ceil_div(rows, d::kBlock), d::kBlock, 0, s>>>(rows, width, data, cols, x, y);
  return check_launch("ell_kernel launch");
}

template <typename T>
int fill(uint64_t n, T *v, T value, void *stream) {
  if (n == 0) return ok();
  if (!v) return fail(MFP_ERROR_INVALID_VALUE, "null vector");
  const uint32_t grid = (uint32_t)std::min<uint64_t>(ceil_div(n, 512), 148u * 16u);
  d::fill_kernel<T><<<grid, 512, 0, as_stream(stream)>>>(n, v, value);
  return check_launch("fill_kernel launch");
}

// Launches that follow another launch of the same call may start early
// (programmatic dependent launch): their CTAs are placed while the preceding
// kernel drains and wait for it in griddep_wait() before touching its output.
#ifndef MFP_PDL
#define MFP_PDL 1
#endif
template <typename... KArgs, typename... Args>
cudaError_t launch_after(void (*k)(KArgs...), uint32_t grid, cudaStream_t s, Args &&...args) {
  if (!MFP_PDL) {
    k<<<grid, d::kBlock, 0, s>>>(std::forward<Args>(args)...);
    return cudaGetLastError();
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(d::kBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}


template <typename T, bool ACCUM = false>
int coo_spmv(uint32_t rows, uint32_t nnz, const T *data, const uint32_t *cols, const uint32_t *rids,
             const T *x, T *y, void *ws, size_t ws_bytes, void *stream, const uint16_t *rel = nullptr,
             const uint32_t *tile_base = nullptr, const uint8_t *rel8 = nullptr, bool wide = false) {
  if (rows == 0) return ok();
  if (!y) return fail(MFP_ERROR_INVALID_VALUE, "null y");
  if (nnz == 0) return ACCUM ? ok() : fill<T>(rows, y, T(0), stream);
  if (!data || !cols || !rids || !x) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  if (!ws || ws_bytes < coo_ws_bytes(nnz))
    return fail(MFP_ERROR_INVALID_VALUE, "COO workspace of %zu bytes needed, %zu given", coo_ws_bytes(nnz), ws_bytes);
  if (!aligned16(ws)) return fail(MFP_ERROR_INVALID_VALUE, "COO workspace must be 16-byte aligned");
  const uint32_t n_wt = ceil_div(nnz, d::kWarpTile);
  auto *hdr = static_cast<d::coo_ws_header *>(ws);
  unsigned char *base = static_cast<unsigned char *>(ws) + sizeof(d::coo_ws_header);
  d::coo_carry<T> cw;
  cw.head = reinterpret_cast<T *>(base);
  cw.tail = reinterpret_cast<T *>(base + (size_t)n_wt * 8u);
  cw.flags = reinterpret_cast<uint32_t *>(base + (size_t)n_wt * 16u);
  cw.tail_row = cw.flags + n_wt;
  const uint32_t grid = ceil_div(n_wt, d::kBlock / 32u);
  const int vec = vec_level(data, cols, rids);
  cudaStream_t s = as_stream(stream);
  // compact 8- or 16-bit rows (handles) on 32-byte-aligned arrays
  const bool r8 = rel8 && tile_base && vec == 2 && aligned16(rel8);
  const bool r16 = !r8 && rel && tile_base && vec == 2 && aligned16(rel);
  auto k = r8    ? (wide ? d::coo_warp_kernel<T, 2, ACCUM, false, true, true>
                         : d::coo_warp_kernel<T, 2, ACCUM, false, true>)
           : r16 ? d::coo_warp_kernel<T, 2, ACCUM, true>
                    : (vec == 2 ? d::coo_warp_kernel<T, 2, ACCUM>
                                : (vec == 1 ? d::coo_warp_kernel<T, 1, ACCUM> : d::coo_warp_kernel<T, 0, ACCUM>));
  if (!r16) rel = nullptr;
  if (!r8) rel8 = nullptr;
  if (!r8 && !r16) tile_base = nullptr;
  // the accumulating warp pass (hybrid tail) follows the ELL launch of the same call
  cudaError_t e;
  if (ACCUM)
    e = launch_after(k, grid, s, rows, nnz, data, cols, rids, x, y, cw, hdr, rel, tile_base, rel8);
  else {
    k<<<grid, d::kBlock, 0, s>>>(rows, nnz, data, cols, rids, x, y, cw, hdr, rel, tile_base, rel8);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return cuda_fail(e, "coo_warp_kernel launch");
  // the fix-up pass finishes rows that cross tiles and, without ACCUM, zeroes
  // the empty rows before the first and after the last row with elements
  if (n_wt > 1 || !ACCUM) {
    uint32_t fgrid = ceil_div(n_wt, d::kBlock);
    if (!ACCUM) fgrid = std::max(fgrid, std::min(ceil_div(rows, d::kBlock * 8u), 148u * 4u));
    e = launch_after(d::coo_fixup_kernel<T, ACCUM>, fgrid, s, n_wt, rows, cw, (const d::coo_ws_header *)hdr, y);
    if (e != cudaSuccess) return cuda_fail(e, "coo_fixup_kernel launch");
  }
  return ok();
}

// The warp-tile CSR (CSR vector on short rows): warp pass + the COO fix-up.
template <typename T>
int csr_tile_spmv(const mfp_csr_plan *plan, const T *data, const uint32_t *cols, const uint32_t *rp, const T *x,
                  T *y, cudaStream_t s) {
  const uint32_t nnz = plan->nnz, rows = plan->rows;
  const uint32_t n_wt = ceil_div(nnz, d::kWarpTile);
  auto *hdr = static_cast<d::coo_ws_header *>(plan->tile_ws);
  unsigned char *base = static_cast<unsigned char *>(plan->tile_ws) + sizeof(d::coo_ws_header);
  d::coo_carry<T> cw;
  cw.head = reinterpret_cast<T *>(base);
  cw.tail = reinterpret_cast<T *>(base + (size_t)n_wt * 8u);
  cw.flags = reinterpret_cast<uint32_t *>(base + (size_t)n_wt * 16u);
  cw.tail_row = cw.flags + n_wt;
  const uint32_t grid = ceil_div(n_wt, d::kBlock / 32u);
  const int vec = vec_level(data, cols);
  // 64 row starts per round trip below a mean row length of 8 (power-law 4M
  // 0.177 -> 0.175 ms; 32 stays faster for the stencil and banded matrices)
  const bool wide = (uint64_t)nnz < 8ull * rows;
  auto k = wide ? (vec == 2 ? d::csr_tile_kernel<T, 2, true>
                            : (vec == 1 ? d::csr_tile_kernel<T, 1, true> : d::csr_tile_kernel<T, 0, true>))
                : (vec == 2 ? d::csr_tile_kernel<T, 2> : (vec == 1 ? d::csr_tile_kernel<T, 1> : d::csr_tile_kernel<T, 0>));
  k<<<grid, d::kBlock, 0, s>>>(rows, nnz, data, cols, rp, plan->tile_prev, x, y, cw, hdr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "csr_tile_kernel launch");
  const uint32_t fgrid = std::max(ceil_div(n_wt, d::kBlock), std::min(ceil_div(rows, d::kBlock * 8u), 148u * 4u));
  e = launch_after(d::coo_fixup_kernel<T, false>, fgrid, s, n_wt, rows, cw, (const d::coo_ws_header *)hdr, y);
  if (e != cudaSuccess) return cuda_fail(e, "coo_fixup_kernel launch");
  return ok();
}

template <typename T, int VEC, bool XWIN, bool UNSORTED = false, bool R16 = false>
int scoo_launch(uint32_t grid, size_t dyn, cudaStream_t s, uint32_t rows, uint32_t slice, const T *v,
                const uint32_t *ci, const uint32_t *ri, const uint32_t *sp, const uint32_t *win, uint32_t maxw,
                const uint32_t *order, const T *x, T *y, const uint16_t *rel = nullptr) {
  if (UNSORTED) {
    auto k = d::scoo_unsorted_kernel<T, XWIN>;
    if (dyn > 48 * 1024 - sizeof(d::scoo_smem_static<T>)) {
      const int st = ensure_dyn_smem((const void *)k, dyn, "scoo_kernel");
      if (st) return st;
    }
    k<<<grid, d::kBlock, dyn, s>>>(rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
  } else {
    auto k = d::scoo_kernel<T, VEC, XWIN, R16>;
    if (dyn > 48 * 1024 - sizeof(d::scoo_smem_static<T>)) {
      const int st = ensure_dyn_smem((const void *)k, dyn, "scoo_kernel");
      if (st) return st;
    }
    k<<<grid, d::kBlock, dyn, s>>>(rows, slice, v, ci, ri, sp, win, maxw, order, x, y, rel);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(MFP_ERROR_CUDA, "scoo_kernel launch (grid %u, %zu dynamic bytes): %s", grid, dyn, cudaGetErrorString(e));
  return ok();
}

template <typename T, bool UNSORTED = false>
int scoo_spmv(uint32_t rows, uint32_t slices, uint32_t slice, const T *v, const uint32_t *ci,
              const uint32_t *ri, const uint32_t *sp, const uint32_t *win, uint32_t maxw, const uint32_t *order,
              const T *x, T *y, void *stream, const uint16_t *rel = nullptr) {
  if (rows == 0) return ok();
  // values / c_index / r_index may be NULL only when every slice is empty
  if (!y || !sp || !x) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  if (slice == 0 || (uint64_t)slice * slices < rows) return fail(MFP_ERROR_INVALID_VALUE, "slices do not cover the rows");
  const size_t acc_bytes = (size_t)((slice + 3u) & ~3u) * sizeof(T);
  if (win == nullptr) maxw = 0;
  const size_t dyn = acc_bytes + (size_t)maxw * sizeof(T);
  if (dyn + sizeof(d::scoo_smem_static<T>) > 227 * 1024)
    return fail(MFP_ERROR_NOT_SUPPORTED, "slice_size %u / window %u too large for shared memory", slice, maxw);
  const int vec = vec_level(v, ci, ri);
  cudaStream_t s = as_stream(stream);
  if (UNSORTED) {
    if (win) return scoo_launch<T, 0, true, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
    return scoo_launch<T, 0, false, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
  }
  if (vec == 2 && rel && aligned16(rel)) {  // compact 16-bit rows (handles)
    if (win)
      return scoo_launch<T, 2, true, false, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y,
                                                  rel);
    return scoo_launch<T, 2, false, false, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y,
                                                 rel);
  }
  if (vec == 2) {
    if (win) return scoo_launch<T, 2, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
    return scoo_launch<T, 2, false>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
  }
  if (vec == 1) {
    if (win) return scoo_launch<T, 1, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
    return scoo_launch<T, 1, false>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
  }
  if (win) return scoo_launch<T, 0, true>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
  return scoo_launch<T, 0, false>(slices, dyn, s, rows, slice, v, ci, ri, sp, win, maxw, order, x, y);
}

// Pipelined reduced-precision kernel: CAP elements per stage, S stages.  A
// stage of the defaults holds a 256-row block of up to 32 elements per row
// (16-bit indices) in about 35 KB; three CTAs share an SM.
#ifndef MFP_LOWP_CAP16
#define MFP_LOWP_CAP16 8448
#endif
#ifndef MFP_LOWP_CAP32
#define MFP_LOWP_CAP32 5632
#endif
#ifndef MFP_LOWP_STAGES
#define MFP_LOWP_STAGES 2
#endif
#ifndef MFP_LOWP_TMA
#define MFP_LOWP_TMA 1
#endif

template <int VT, bool D16>
int lowp_tma_launch(const d::lowp_args<VT, D16> &A, uint32_t nnz, cudaStream_t s) {
  constexpr uint32_t CAP = D16 ? MFP_LOWP_CAP16 : MFP_LOWP_CAP32;
  constexpr uint32_t S = MFP_LOWP_STAGES;
  static_assert(CAP % 8 == 0 && CAP >= 8, "stage capacity must be a multiple of 8 elements");
  auto k = d::lowp_tma_kernel<VT, D16, CAP, S>;
  const size_t dyn = d::lowp_pipe_bytes<D16, CAP, S>();
  int st = ensure_dyn_smem((const void *)k, dyn, "lowp_tma_kernel");
  if (st) return st;
  uint32_t grid = 0;
  if ((st = persistent_grid((const void *)k, (int)d::kLowpThreads, dyn, &grid))) return st;
  grid = std::min(grid, ceil_div(A.n_rows, d::kLowpRows));
  k<<<grid, d::kLowpThreads, dyn, s>>>(A, nnz);
  return check_launch("lowp_tma_kernel launch");
}

// long_rows: the matrix has rows longer than kLowpTmaMaxRow elements; they go
// to the row-block kernel, whose warps share long rows (the pipelined kernel
// sums each row in one thread).  Handles know it; the raw entry point does not.
constexpr uint32_t kLowpTmaMaxRow = 1024;
int lowp_spmv(int vt, uint32_t rows, uint32_t nnz, const uint32_t *rp, const uint16_t *q, const float *scale,
              const uint32_t *cols, const uint16_t *delta, const uint32_t *base, const float *x, float *y,
              void *stream, bool long_rows = false) {
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (rows == 0) return ok();
  if (rows > 0xffffff00u) return fail(MFP_ERROR_TOO_LARGE, "too many rows");
  if (!rp || !scale || !y || (nnz && (!q || !x || (!cols && !(delta && base)))))
    return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  const bool d16 = cols == nullptr;
  const bool vec = aligned16(q) && (d16 ? aligned16(delta) : aligned16(cols));
  cudaStream_t s = as_stream(stream);
  // TMA bulk copies need 16-byte-aligned sources: values, indices and row_ptr
  if (MFP_LOWP_TMA && nnz && vec && aligned16(rp) && !long_rows) {
    if (vt == MFP_BF16)
      return d16 ? lowp_tma_launch<2, true>({rows, rp, q, scale, cols, delta, base, x, y}, nnz, s)
                 : lowp_tma_launch<2, false>({rows, rp, q, scale, cols, delta, base, x, y}, nnz, s);
    return d16 ? lowp_tma_launch<3, true>({rows, rp, q, scale, cols, delta, base, x, y}, nnz, s)
               : lowp_tma_launch<3, false>({rows, rp, q, scale, cols, delta, base, x, y}, nnz, s);
  }
  const uint32_t grid = ceil_div(rows, d::kBlock);
#define MFP_LOWP(VT, D16, VEC)                                                     \
  {                                                                                \
    d::lowp_args<VT, D16> A{rows, rp, q, scale, cols, delta, base, x, y};          \
    d::lowp_kernel<VT, D16, VEC><<<grid, d::kBlock, 0, s>>>(A);                    \
  }
  if (vt == MFP_BF16) {
    if (d16) {
      if (vec) MFP_LOWP(2, true, true) else MFP_LOWP(2, true, false)
    } else {
      if (vec) MFP_LOWP(2, false, true) else MFP_LOWP(2, false, false)
    }
  } else {
    if (d16) {
      if (vec) MFP_LOWP(3, true, true) else MFP_LOWP(3, true, false)
    } else {
      if (vec) MFP_LOWP(3, false, true) else MFP_LOWP(3, false, false)
    }
  }
#undef MFP_LOWP
  return check_launch("lowp_kernel launch");
}

// Runs of 8 consecutive x entries read with 16-byte loads where a lane's rows
// share a column offset (1), or always 8 gathers (0).
#ifndef MFP_LOWP_XRUN
#define MFP_LOWP_XRUN 1
#endif
// The 16-bit ELL kernel's VEC path (8 consecutive rows per thread, 16-byte
// loads) when the layout allows it (1), or always the lane-interleaved path (0).
#ifndef MFP_LOWP_ELL_VEC
#define MFP_LOWP_ELL_VEC 1
#endif
int lowp_ell_spmv(int vt, uint32_t rows, uint32_t cols_n, uint32_t width, const uint16_t *q, const float *scale,
                  const uint32_t *cols, const uint16_t *off, const float *x, float *y, void *stream) {
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (rows == 0) return ok();
  if (!scale || !y || (width && (!q || !x || (!cols && !off)))) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  const bool d16 = cols == nullptr;
  const bool vec = MFP_LOWP_ELL_VEC && rows % 8 == 0 && aligned16(q) && (d16 ? aligned16(off) : aligned16(cols));
  cudaStream_t s = as_stream(stream);
  const uint32_t grid = ceil_div(ceil_div(rows, 8), d::kBlock);
#define MFP_LELL(VT, D16)                                                                         \
  {                                                                                               \
    d::lowp_ell_args<VT, D16> A{rows, width, cols_n, q, scale, cols, off, x, y};                  \
    if (MFP_LOWP_XRUN && vec && D16 && aligned16(x) && aligned16(y) && aligned16(scale))          \
      d::lowp_ell_kernel<VT, D16, true, true><<<grid, d::kBlock, 0, s>>>(A);                      \
    else if (vec)                                                                                 \
      d::lowp_ell_kernel<VT, D16, true><<<grid, d::kBlock, 0, s>>>(A);                            \
    else                                                                                          \
      d::lowp_ell_kernel<VT, D16, false><<<grid, d::kBlock, 0, s>>>(A);                           \
  }
  if (vt == MFP_BF16) {
    if (d16) MFP_LELL(2, true) else MFP_LELL(2, false)
  } else {
    if (d16) MFP_LELL(3, true) else MFP_LELL(3, false)
  }
#undef MFP_LELL
  return check_launch("lowp_ell_kernel launch");
}

// Hybrid: the ELL kernel writes every row's ELL part, then the tile-based COO
// kernel adds the tail (elements past the ELL width) row by row.
template <typename T>
int hyb_spmv(uint32_t rows, uint32_t width, const T *ed, const uint32_t *ec, uint32_t cnnz, const T *cd,
             const uint32_t *cc, const uint32_t *cr, const T *x, T *y, void *ws, size_t ws_bytes, void *stream,
             const uint16_t *rel = nullptr, const uint32_t *tile_base = nullptr, const uint8_t *rel8 = nullptr,
             bool wide = false) {
  if (rows == 0) return ok();
  if (!y || !x || (width && (!ed || !ec)) || (cnnz && (!cd || !cc || !cr)))
    return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  int st = ell_spmv<T>(rows, width, ed, ec, x, y, stream);
  if (st) return st;
  return coo_spmv<T, true>(rows, cnnz, cd, cc, cr, x, y, ws, ws_bytes, stream, rel, tile_base, rel8, wide);
}
}  // namespace

extern "C" {

int mfp_get_device_info(int device, mfp_device_info *out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  cudaDeviceProp p{};
  CUDA_TRY(cudaGetDeviceProperties(&p, device), "cudaGetDeviceProperties");
  out->device = device;
  out->sm_count = p.multiProcessorCount;
  out->shared_mem_per_block = p.sharedMemPerBlock;
  out->shared_mem_optin = p.sharedMemPerBlockOptin;
  out->l2_bytes = (uint64_t)p.l2CacheSize;
  out->global_mem_bytes = p.totalGlobalMem;
  out->cc_major = p.major;
  out->cc_minor = p.minor;
  return ok();
}

int mfp_csr_spmv_f32(const mfp_csr_plan *p, const float *a, const uint32_t *c, const uint32_t *rp, const float *x,
                     float *y, void *s) {
  return csr_spmv<float>(p, a, c, rp, x, y, s);
}
int mfp_csr_spmv_f64(const mfp_csr_plan *p, const double *a, const uint32_t *c, const uint32_t *rp,
                     const double *x, double *y, void *s) {
  return csr_spmv<double>(p, a, c, rp, x, y, s);
}
int mfp_ell_spmv_f32(uint32_t rows, uint32_t, uint32_t w, const float *a, const uint32_t *c, const float *x,
                     float *y, void *s) {
  return ell_spmv<float>(rows, w, a, c, x, y, s);
}
int mfp_ell_spmv_f64(uint32_t rows, uint32_t, uint32_t w, const double *a, const uint32_t *c, const double *x,
                     double *y, void *s) {
  return ell_spmv<double>(rows, w, a, c, x, y, s);
}
int mfp_coo_workspace_bytes(uint32_t, uint32_t nnz, size_t *bytes) {
  if (!bytes) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *bytes = coo_ws_bytes(nnz);
  return ok();
}
int mfp_coo_spmv_f32(uint32_t rows, uint32_t, uint32_t nnz, const float *a, const uint32_t *c, const uint32_t *r,
                     const float *x, float *y, void *ws, size_t wsb, void *s) {
  return coo_spmv<float>(rows, nnz, a, c, r, x, y, ws, wsb, s);
}
int mfp_coo_spmv_f64(uint32_t rows, uint32_t, uint32_t nnz, const double *a, const uint32_t *c, const uint32_t *r,
                     const double *x, double *y, void *ws, size_t wsb, void *s) {
  return coo_spmv<double>(rows, nnz, a, c, r, x, y, ws, wsb, s);
}
int mfp_workspace_error(const void *ws, uint32_t *error) {
  if (!ws || !error) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  d::coo_ws_header h{};
  CUDA_TRY(cudaMemcpy(&h, ws, sizeof(h), cudaMemcpyDeviceToHost), "cudaMemcpy D2H");
  *error = h.error;
  return ok();
}
int mfp_scoo_slice_order(uint32_t slices, const uint32_t *sp, uint32_t *order) {
  if (slices && (!sp || !order)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  for (uint32_t k = 0; k < slices; ++k) order[k] = k;
  auto cnt = [&](uint32_t k) { return sp[k + 1] >= sp[k] ? sp[k + 1] - sp[k] : 0u; };
  std::stable_sort(order, order + slices, [&](uint32_t a, uint32_t b) { return cnt(a) > cnt(b); });
  return ok();
}
int mfp_scoo_spmv_f32(uint32_t rows, uint32_t, uint32_t slices, uint32_t slice, const float *v, const uint32_t *ci,
                      const uint32_t *ri, const uint32_t *sp, const uint32_t *win, uint32_t maxw,
                      const uint32_t *order, const float *x, float *y, void *s) {
  return scoo_spmv<float>(rows, slices, slice, v, ci, ri, sp, win, maxw, order, x, y, s);
}
int mfp_scoo_spmv_f64(uint32_t rows, uint32_t, uint32_t slices, uint32_t slice, const double *v, const uint32_t *ci,
                      const uint32_t *ri, const uint32_t *sp, const uint32_t *win, uint32_t maxw,
                      const uint32_t *order, const double *x, double *y, void *s) {
  return scoo_spmv<double>(rows, slices, slice, v, ci, ri, sp, win, maxw, order, x, y, s);
}
int mfp_scoo_spmv_unsorted_f32(uint32_t rows, uint32_t, uint32_t slices, uint32_t slice, const float *v,
                               const uint32_t *ci, const uint32_t *ri, const uint32_t *sp, const uint32_t *win,
                               uint32_t maxw, const uint32_t *order, const float *x, float *y, void *s) {
  return scoo_spmv<float, true>(rows, slices, slice, v, ci, ri, sp, win, maxw, order, x, y, s);
}
int mfp_scoo_spmv_unsorted_f64(uint32_t rows, uint32_t, uint32_t slices, uint32_t slice, const double *v,
                               const uint32_t *ci, const uint32_t *ri, const uint32_t *sp, const uint32_t *win,
                               uint32_t maxw, const uint32_t *order, const double *x, double *y, void *s) {
  return scoo_spmv<double, true>(rows, slices, slice, v, ci, ri, sp, win, maxw, order, x, y, s);
}
int mfp_lowp_spmv(int vt, uint32_t rows, uint32_t, uint32_t nnz, const uint32_t *rp, const uint16_t *q,
                  const float *scale, const uint32_t *cols, const uint16_t *delta, const uint32_t *base,
                  const float *x, float *y, void *s) {
  return lowp_spmv(vt, rows, nnz, rp, q, scale, cols, delta, base, x, y, s);
}
int mfp_lowp_ell_spmv(int vt, uint32_t rows, uint32_t ncols, uint32_t width, const uint16_t *q, const float *scale,
                      const uint32_t *cols, const uint16_t *off, const float *x, float *y, void *s) {
  return lowp_ell_spmv(vt, rows, ncols, width, q, scale, cols, off, x, y, s);
}
}  // extern "C"
template <int MODE, int XPATH>
int probe_launch(uint32_t nnz, const float *v, const uint32_t *c, const float *x, float *out, size_t out_len,
                 cudaStream_t s) {
  auto k = d::probe_loads_kernel<MODE, XPATH>;
  uint32_t grid = 0;
  int st = persistent_grid((const void *)k, d::kProbeBlock, 0, &grid);
  if (st) return st;
  if (out_len < grid) return fail(MFP_ERROR_INVALID_VALUE, "probe output needs %u floats, %zu given", grid, out_len);
  k<<<grid, d::kProbeBlock, 0, s>>>(nnz, v, c, x, out);
  return check_launch("probe_loads_kernel launch");
}
// x as a 2-D tensor of n/4 rows of 4 floats (16-byte rows; x 16-byte aligned,
// n a multiple of 4), box one row high: the map tile::gather4 needs.
int x_rows_map(const float *x, uint32_t n, CUtensorMap *map) {
  using encode_fn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static encode_fn encode = nullptr;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> g(mu);
    if (!encode) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q{};
      const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
      if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
        return fail(MFP_ERROR_CUDA, "cuTensorMapEncodeTiled entry point not found");
      encode = reinterpret_cast<encode_fn>(fn);
    }
  }
  if (!aligned16(x) || n % 4 != 0 || n < 4) return fail(MFP_ERROR_INVALID_VALUE, "x must be 16-byte aligned with n %% 4 == 0");
  const cuuint64_t dims[2] = {4, n / 4};
  const cuuint64_t strides[1] = {16};
  const cuuint32_t box[2] = {4, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(x), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MFP_ERROR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return ok();
}
template <int MODE>
int probe_g4_launch(uint32_t nnz, uint32_t n_x, const uint32_t *c, const float *x, float *out, size_t out_len,
                    cudaStream_t s) {
  CUtensorMap map;
  int st = x_rows_map(x, n_x, &map);
  if (st) return st;
  auto k = d::probe_gather4_kernel<MODE>;
  if ((st = ensure_dyn_smem((const void *)k, d::kG4DynBytes, "probe_gather4_kernel"))) return st;
  uint32_t grid = 0;
  if ((st = persistent_grid((const void *)k, d::kG4Warps * 32, d::kG4DynBytes, &grid))) return st;
  if (out_len < grid) return fail(MFP_ERROR_INVALID_VALUE, "probe output needs %u floats, %zu given", grid, out_len);
  k<<<grid, d::kG4Warps * 32, d::kG4DynBytes, s>>>(nnz, c, x, map, out);
  return check_launch("probe_gather4_kernel launch");
}
extern "C" {
int mfp_probe_spmv_gather4(int mode, uint32_t nnz, uint32_t n_x, const uint32_t *col_ids, const float *x, float *out,
                           size_t out_len, void *stream) {
  if (mode != 4 && mode != 5) return fail(MFP_ERROR_INVALID_VALUE, "mode must be 4 or 5");
  if (nnz == 0) return ok();
  if (!col_ids || !x || !out) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  if (!aligned16(col_ids)) return fail(MFP_ERROR_INVALID_VALUE, "the probe needs 16-byte-aligned arrays");
  cudaStream_t s = as_stream(stream);
  return mode == 4 ? probe_g4_launch<4>(nnz, n_x, col_ids, x, out, out_len, s)
                   : probe_g4_launch<5>(nnz, n_x, col_ids, x, out, out_len, s);
}
int mfp_probe_spmv_loads(int mode, int x_path, uint32_t nnz, const float *values, const uint32_t *col_ids,
                         const float *x, float *out, size_t out_len, void *stream) {
  if (mode < 0 || mode > 3 || x_path < 0 || x_path > 2) return fail(MFP_ERROR_INVALID_VALUE, "mode / x_path out of range");
  if (nnz == 0) return ok();
  if (!col_ids || !out || ((mode == 0 || mode == 2) && !values) || (mode != 0 && !x))
    return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  if (!aligned16(col_ids) || ((mode == 0 || mode == 2) && !aligned16(values)))
    return fail(MFP_ERROR_INVALID_VALUE, "the probe needs 16-byte-aligned arrays");
  cudaStream_t s = as_stream(stream);
  if (mode == 0) return probe_launch<0, 0>(nnz, values, col_ids, x, out, out_len, s);
  if (mode == 1) {
    if (x_path == 0) return probe_launch<1, 0>(nnz, values, col_ids, x, out, out_len, s);
    if (x_path == 1) return probe_launch<1, 1>(nnz, values, col_ids, x, out, out_len, s);
    return probe_launch<1, 2>(nnz, values, col_ids, x, out, out_len, s);
  }
  if (mode == 3) return probe_launch<3, 0>(nnz, values, col_ids, x, out, out_len, s);
  if (x_path == 0) return probe_launch<2, 0>(nnz, values, col_ids, x, out, out_len, s);
  if (x_path == 1) return probe_launch<2, 1>(nnz, values, col_ids, x, out, out_len, s);
  return probe_launch<2, 2>(nnz, values, col_ids, x, out, out_len, s);
}
int mfp_lowp_error(int device, int clear, uint32_t *error) {
  if (!error) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  int prev = 0;
  CUDA_TRY(cudaGetDevice(&prev), "cudaGetDevice");
  CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
  cudaError_t e = cudaMemcpyFromSymbol(error, d::g_lowp_error, sizeof(uint32_t));
  if (e == cudaSuccess && clear) {
    const uint32_t zero = 0;
    e = cudaMemcpyToSymbol(d::g_lowp_error, &zero, sizeof(uint32_t));
  }
  cudaSetDevice(prev);
  if (e != cudaSuccess) return cuda_fail(e, "lowp error word");
  return ok();
}
int mfp_hybrid_workspace_bytes(uint32_t rows, uint32_t coo_nnz, size_t *bytes) {
  if (!bytes) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *bytes = coo_ws_bytes(coo_nnz);
  return ok();
}
int mfp_hybrid_spmv_f32(uint32_t rows, uint32_t, uint32_t w, const float *ed, const uint32_t *ec, uint32_t cn,
                        const float *cd, const uint32_t *cc, const uint32_t *cr, const float *x, float *y, void *ws,
                        size_t wsb, void *s) {
  return hyb_spmv<float>(rows, w, ed, ec, cn, cd, cc, cr, x, y, ws, wsb, s);
}
int mfp_hybrid_spmv_f64(uint32_t rows, uint32_t, uint32_t w, const double *ed, const uint32_t *ec, uint32_t cn,
                        const double *cd, const uint32_t *cc, const uint32_t *cr, const double *x, double *y,
                        void *ws, size_t wsb, void *s) {
  return hyb_spmv<double>(rows, w, ed, ec, cn, cd, cc, cr, x, y, ws, wsb, s);
}
int mfp_fill_f32(uint64_t n, float *v, float value, void *s) { return fill<float>(n, v, value, s); }
int mfp_fill_f64(uint64_t n, double *v, double value, void *s) { return fill<double>(n, v, value, s); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Device-resident matrices
// ---------------------------------------------------------------------------
struct mfp_matrix {
  int format = 0, value_type = 0, device = 0;
  uint32_t rows = 0, cols = 0;
  uint64_t nnz = 0;
  std::vector<void *> allocs;
  size_t device_bytes = 0;
  uint64_t format_bytes = 0;
  // arrays (meaning per format)
  void *vals = nullptr;
  uint32_t *cols_a = nullptr;
  uint32_t *rows_a = nullptr;   // CSR row_ptr, COO/SCOO row ids
  uint32_t *aux = nullptr;      // SCOO slices_ptr
  uint32_t *win = nullptr;      // SCOO x windows
  uint32_t *order = nullptr;    // SCOO slices, heaviest first
  void *vals2 = nullptr;        // HYB COO tail
  uint32_t *cols2 = nullptr, *rows2 = nullptr;
  uint32_t width = 0, coo_nnz = 0, slices = 0, slice_size = 0, max_window = 0;
  mfp_csr_plan *plan = nullptr;
  void *ws = nullptr;
  size_t ws_bytes = 0;
  // compact rows (COO, the hybrid's tail, row-ordered SCOO): 16-bit (rel) or
  // 8-bit (rel8) offsets from each 256-element tile's first row (tile_base),
  // 16-bit from the slice's first row for SCOO; NULL when some offset needs
  // more than 16 bits
  uint16_t *rel = nullptr;
  uint32_t *tile_base = nullptr;
  uint8_t *rel8 = nullptr;  // COO / hybrid tail: 8-bit offsets (tiles of at most 256 rows)
  uint32_t wide_tiles = 0;  // with rel8: tiles spanning more rows, which read rows_a / rows2
  void *dx = nullptr, *dy = nullptr;  // staging for the host-buffer call
  // second staging pair, copy streams and events of the pipelined host-buffer
  // call (made on its first use)
  void *dx2 = nullptr, *dy2 = nullptr;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_start = nullptr, ev_in[2] = {}, ev_k[2] = {}, ev_out[2] = {};
  int lowp_vt = 0;                    // reduced-precision CSR: MFP_BF16 / MFP_F16
  float *scale = nullptr;
  uint16_t *delta = nullptr;          // 16-bit column deltas (else cols_a)
  uint32_t *base = nullptr;
  bool rows_unsorted = false;         // SCOO in the sort_cols layout
  bool long_rows = false;             // reduced-precision CSR: a row longer than kLowpTmaMaxRow
};

namespace {

template <typename T>
int track(mfp_matrix *m, T **p, size_t count) {
  int st = dmalloc(p, count, &m->device_bytes);
  if (!st && *p) m->allocs.push_back(*p);
  return st;
}
template <typename T>
int track_upload(mfp_matrix *m, T **p, const T *host, size_t count) {
  int st = track(m, p, count);
  if (st) return st;
  if (count) CUDA_TRY(cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  return MFP_SUCCESS;
}
int track_upload_bytes(mfp_matrix *m, void **p, const void *host, size_t bytes) {
  unsigned char *q = nullptr;
  int st = track_upload(m, &q, static_cast<const unsigned char *>(host), bytes);
  *p = q;
  return st;
}
// Compact rows for the COO-family handles: 8- or 16-bit offsets built on the
// device from the uploaded 32-bit rows.  Kept only when every offset fits; the
// format's byte count then charges 1 or 2 bytes per row id (and 4 per tile
// base).
// the fit flag of the compact-row conversion (one conversion at a time)
__device__ uint32_t g_rows16_flag[2];
std::mutex g_rows16_mu;

int attach_compact_rows(mfp_matrix *m) {
  const bool coo = m->format == MFP_FORMAT_COO, hyb = m->format == MFP_FORMAT_HYBRID;
  const bool scoo = m->format == MFP_FORMAT_SCOO && !m->rows_unsorted;
  const uint32_t n = coo ? (uint32_t)m->nnz : hyb ? m->coo_nnz : scoo ? (uint32_t)m->nnz : 0u;
  const uint32_t *rows = hyb ? m->rows2 : m->rows_a;
  if (!MFP_COMPACT_ROWS || n == 0 || !rows || (scoo && m->slice_size > 65536u)) return ok();
  const uint32_t tiles = scoo ? 0u : ceil_div(n, d::kWarpTile);
  const uint32_t warp_grid = ceil_div(tiles, d::kBlock / 32u);
  int st = 0;
  uint32_t hflag[2] = {0, 0};
  std::lock_guard<std::mutex> g(g_rows16_mu);
  uint32_t *flag = nullptr;
  const uint32_t zero[2] = {0, 0};
  if (cudaGetSymbolAddress(reinterpret_cast<void **>(&flag), g_rows16_flag) != cudaSuccess ||
      cudaMemcpy(flag, zero, sizeof(zero), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(MFP_ERROR_CUDA, "compact rows: %s", cudaGetErrorString(cudaGetLastError()));
  // the offsets' width: SCOO 16 bits (from the slice's first row); COO 8 bits
  // when at most one tile in 8 spans more than 256 rows (those read the
  // 32-bit rows; FP32 only: with FP64 values such tiles cost 3% on the
  // power-law hybrid's tail), else 16 bits when every offset fits, else none
  uint32_t w = 2;
  if (!scoo) {
    d::coo_rows_span_kernel<<<warp_grid, d::kBlock>>>(n, rows, flag);
    if (cudaMemcpy(hflag, flag, sizeof(hflag), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail(MFP_ERROR_CUDA, "compact rows: %s", cudaGetErrorString(cudaGetLastError()));
    if (MFP_COMPACT_ROWS8 && m->rows <= d::kWideTile && hflag[1] <= tiles / 8u &&
        (hflag[1] == 0 || m->value_type == MFP_F32))
      w = 1;
    else if (hflag[0] & 1u) return ok();  // 32-bit rows
  }
  // one allocation: the offsets, then (16-byte aligned) the tile bases
  const size_t rel_bytes = ((size_t)n * w + 15) & ~(size_t)15;
  unsigned char *blk = nullptr;
  if ((st = dmalloc(&blk, rel_bytes + (size_t)tiles * 4, nullptr))) return st;
  uint32_t *base = tiles ? reinterpret_cast<uint32_t *>(blk + rel_bytes) : nullptr;
  if (scoo)
    d::scoo_rows16_kernel<<<m->slices, d::kBlock>>>(m->slice_size, m->aux, rows, reinterpret_cast<uint16_t *>(blk),
                                                     flag);
  else if (w == 1)
    d::coo_rows8_kernel<<<warp_grid, d::kBlock>>>(n, rows, base, blk);
  else
    d::coo_rows16_kernel<<<ceil_div(n, d::kBlock), d::kBlock>>>(n, rows, base, reinterpret_cast<uint16_t *>(blk));
  if (cudaMemcpy(hflag, flag, sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = fail(MFP_ERROR_CUDA, "compact rows: %s", cudaGetErrorString(cudaGetLastError()));
  if (st || (scoo && (hflag[0] & 1u))) {  // an offset does not fit: 32-bit rows
    cudaFree(blk);
    return st;
  }
  if (w == 1) m->rel8 = blk, m->wide_tiles = hflag[1];
  else m->rel = reinterpret_cast<uint16_t *>(blk);
  m->tile_base = base;
  m->allocs.push_back(blk);
  m->device_bytes += rel_bytes + (size_t)tiles * 4;
  // bytes a launch reads for the rows: w per element, 4 per tile base, and
  // 4 - w more per element of a wide tile
  m->format_bytes -= (uint64_t)n * (4u - w);
  m->format_bytes += (uint64_t)tiles * 4 + (w == 1 ? (uint64_t)hflag[1] * d::kWarpTile * 3u : 0u);
  return ok();
}

int finish_matrix(mfp_matrix *m, mfp_matrix **out) {
  const size_t vs = value_size(m->value_type);
  {
    const int st0 = attach_compact_rows(m);
    if (st0) {
      mfp_matrix_destroy(m);
      return st0;
    }
  }
  int st = track_upload_bytes(m, &m->dx, nullptr, 0);
  unsigned char *a = nullptr, *b = nullptr;
  if (!st) st = track(m, &a, (size_t)std::max(1u, m->cols) * vs);
  if (!st) st = track(m, &b, (size_t)std::max(1u, m->rows) * vs);
  m->dx = a;
  m->dy = b;
  if (st) {
    mfp_matrix_destroy(m);
    return st;
  }
  *out = m;
  return ok();
}
bool valid_vt(int vt) { return vt == MFP_F32 || vt == MFP_F64; }

int track_bytes(mfp_matrix *m, void **p, size_t bytes) {
  unsigned char *q = nullptr;
  const int st = track(m, &q, bytes);
  *p = q;
  return st;
}

// SCOO x windows ([lo, hi) column range per slice, host copy) and slice order:
// a slice's x window is staged in shared memory when 90% of the windows fit;
// slices launch heaviest first.
int scoo_attach_windows(mfp_matrix *m, const std::vector<uint32_t> &win, const uint32_t *sp_host) {
  const size_t vs = value_size(m->value_type);
  std::vector<uint32_t> widths;
  for (uint32_t s = 0; s < m->slices; ++s)
    if (win[2 * s + 1] > win[2 * s]) widths.push_back(win[2 * s + 1] - win[2 * s]);
  const uint32_t cap = (uint32_t)((m->value_type == MFP_F64 ? 48u : 96u) * 1024u / vs);
  bool use_win = false;
  if (!widths.empty()) {
    std::sort(widths.begin(), widths.end());
    const uint32_t p90 = widths[(widths.size() * 9) / 10];
    if (p90 <= cap) {
      use_win = true;
      m->max_window = std::min(cap, widths.back());
      m->max_window = (m->max_window + 3u) & ~3u;
    }
  }
  int st;
  if (use_win && (st = track_upload(m, &m->win, win.data(), win.size()))) return st;
  std::vector<uint32_t> order(m->slices);
  if ((st = mfp_scoo_slice_order(m->slices, sp_host, order.data())) ||
      (st = track_upload(m, &m->order, order.data(), order.size())))
    return st;
  return MFP_SUCCESS;
}

int check_columns(const uint32_t *c, uint64_t n, uint32_t cols) {
  for (uint64_t i = 0; i < n; ++i)
    if (c[i] >= cols && !(cols == 0 && c[i] == 0))
      return fail(MFP_ERROR_INVALID_VALUE, "column id %u >= cols %u at %llu", c[i], cols, (unsigned long long)i);
  return MFP_SUCCESS;
}

}  // namespace

extern "C" {

int mfp_matrix_destroy(mfp_matrix *m) {
  if (!m) return ok();
  if (m->s_in) cudaStreamSynchronize(m->s_in);
  if (m->s_out) cudaStreamSynchronize(m->s_out);
  for (cudaEvent_t e : {m->ev_start, m->ev_in[0], m->ev_in[1], m->ev_k[0], m->ev_k[1], m->ev_out[0], m->ev_out[1]})
    if (e) cudaEventDestroy(e);
  if (m->s_in) cudaStreamDestroy(m->s_in);
  if (m->s_out) cudaStreamDestroy(m->s_out);
  for (void *p : m->allocs) cudaFree(p);
  mfp_csr_plan_destroy(m->plan);
  delete m;
  return ok();
}

int mfp_matrix_create_csr(int format, int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp,
                          const uint32_t *ci, const void *data, const mfp_csr_config *cfg, mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (format < 0 || format > 2 || !valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad format or value type");
  if (nnz && (!ci || !data)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  int st = check_row_ptr(rows, nnz, rp);
  if (st) return st;
  if ((st = check_columns(ci, nnz, cols))) return st;
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = format;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  const size_t vs = value_size(vt);
  m->format_bytes = (uint64_t)nnz * (vs + 4) + ((uint64_t)rows + 1) * 4 + (uint64_t)cols * vs + (uint64_t)rows * vs;
  if ((st = track_upload_bytes(m, &m->vals, data, (size_t)nnz * vs)) ||
      (st = track_upload(m, &m->cols_a, ci, nnz)) || (st = track_upload(m, &m->rows_a, rp, (size_t)rows + 1)) ||
      (st = mfp_csr_plan_create(rows, cols, nnz, rp, format, cfg, &m->plan))) {
    mfp_matrix_destroy(m);
    return st;
  }
  m->device_bytes += m->plan->device_bytes;
  return finish_matrix(m, out);
}

int mfp_matrix_create_ell(int vt, uint32_t rows, uint32_t cols, uint32_t width, const uint32_t *ec,
                          const void *ed, mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  const uint64_t slots = (uint64_t)rows * width;
  if (slots && (!ec || !ed)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  int st0 = check_columns(ec, slots, cols);
  if (st0) return st0;
  const size_t vs = value_size(vt);
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_ELL;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->width = width;
  // non-padding slots: a padding slot holds column 0 and value 0
  uint64_t nz = 0;
  for (uint64_t i = 0; i < slots; ++i) {
    const bool zero = vt == MFP_F64 ? static_cast<const double *>(ed)[i] == 0.0 : static_cast<const float *>(ed)[i] == 0.0f;
    nz += !(zero && ec[i] == 0);
  }
  m->nnz = nz;
  m->format_bytes = slots * (vs + 4) + (uint64_t)cols * vs + (uint64_t)rows * vs;
  int st;
  if ((st = track_upload_bytes(m, &m->vals, ed, slots * vs)) || (st = track_upload(m, &m->cols_a, ec, slots))) {
    mfp_matrix_destroy(m);
    return st;
  }
  return finish_matrix(m, out);
}

int mfp_matrix_create_coo(int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *cr,
                          const uint32_t *cc, const void *cd, mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (nnz && (!cr || !cc || !cd)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  for (uint32_t i = 0; i < nnz; ++i) {
    if (cr[i] >= rows || cc[i] >= cols) return fail(MFP_ERROR_INVALID_VALUE, "index out of range at element %u", i);
    if (i && cr[i] < cr[i - 1]) return fail(MFP_ERROR_INVALID_VALUE, "COO rows must be sorted (element %u)", i);
  }
  const size_t vs = value_size(vt);
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_COO;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  m->format_bytes = (uint64_t)nnz * (vs + 8) + (uint64_t)cols * vs + (uint64_t)rows * vs;
  m->ws_bytes = coo_ws_bytes(nnz);
  unsigned char *ws = nullptr;
  int st;
  if ((st = track_upload_bytes(m, &m->vals, cd, (size_t)nnz * vs)) || (st = track_upload(m, &m->cols_a, cc, nnz)) ||
      (st = track_upload(m, &m->rows_a, cr, nnz)) || (st = track(m, &ws, m->ws_bytes))) {
    mfp_matrix_destroy(m);
    return st;
  }
  m->ws = ws;
  if (ws && cudaMemset(ws, 0, m->ws_bytes) != cudaSuccess) {
    mfp_matrix_destroy(m);
    return fail(MFP_ERROR_CUDA, "cudaMemset workspace");
  }
  return finish_matrix(m, out);
}

int mfp_matrix_create_scoo(int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const mfp_scoo_params *prm,
                           const uint32_t *ci, const uint32_t *ri, const uint32_t *sp, const void *v,
                           mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (!valid_vt(vt) || !prm || !sp) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  if (nnz && (!ci || !ri || !v)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  bool rows_unsorted = false;
  {
    int st0 = check_columns(ci, nnz, cols);
    if (st0) return st0;
    if ((uint64_t)prm->slice_size * prm->slices_count < rows)
      return fail(MFP_ERROR_INVALID_VALUE, "slices do not cover the rows");
    for (uint32_t s = 0; s < prm->slices_count; ++s) {
      const uint32_t b = sp[s], e = sp[s + 1];
      if (b >= e) continue;
      if (e > nnz) return fail(MFP_ERROR_INVALID_VALUE, "slices_ptr[%u] beyond nnz", s + 1);
      const uint64_t r0 = (uint64_t)s * prm->slice_size, r1 = std::min<uint64_t>(rows, r0 + prm->slice_size);
      for (uint32_t k = b; k < e; ++k) {
        if (ri[k] < r0 || ri[k] >= r1) return fail(MFP_ERROR_INVALID_VALUE, "r_index[%u] outside slice %u", k, s);
        if (k > b && ri[k] < ri[k - 1]) rows_unsorted = true;  // the sort_cols layout
      }
    }
  }
  const size_t vs = value_size(vt);
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_SCOO;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  m->slices = prm->slices_count;
  m->slice_size = prm->slice_size;
  m->rows_unsorted = rows_unsorted;
  m->format_bytes = (uint64_t)nnz * (vs + 8) + ((uint64_t)m->slices + 1) * 4 + (uint64_t)cols * vs + (uint64_t)rows * vs;
  std::vector<uint32_t> win(2 * (size_t)m->slices);
  mfp_scoo_x_windows(nnz, ci, sp, m->slices, win.data());
  int st;
  if ((st = track_upload_bytes(m, &m->vals, v, (size_t)nnz * vs)) || (st = track_upload(m, &m->cols_a, ci, nnz)) ||
      (st = track_upload(m, &m->rows_a, ri, nnz)) || (st = track_upload(m, &m->aux, sp, (size_t)m->slices + 1)) ||
      (st = scoo_attach_windows(m, win, sp))) {
    mfp_matrix_destroy(m);
    return st;
  }
  return finish_matrix(m, out);
}

int mfp_matrix_create_hybrid(int vt, uint32_t rows, uint32_t cols, uint32_t width, const uint32_t *ec,
                             const void *ed, uint32_t cnnz, const uint32_t *cr, const uint32_t *cc, const void *cd,
                             mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  const uint64_t slots = (uint64_t)rows * width;
  if ((slots && (!ec || !ed)) || (cnnz && (!cr || !cc || !cd))) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  for (uint32_t i = 0; i < cnnz; ++i) {
    if (cr[i] >= rows || cc[i] >= cols) return fail(MFP_ERROR_INVALID_VALUE, "tail index out of range at %u", i);
    if (i && cr[i] < cr[i - 1]) return fail(MFP_ERROR_INVALID_VALUE, "tail rows must be sorted (element %u)", i);
  }
  {
    int st0 = check_columns(ec, slots, cols);
    if (st0) return st0;
  }
  const size_t vs = value_size(vt);
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_HYBRID;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->width = width;
  m->coo_nnz = cnnz;
  uint64_t nz = 0;
  for (uint64_t i = 0; i < slots; ++i) {
    const bool zero = vt == MFP_F64 ? static_cast<const double *>(ed)[i] == 0.0 : static_cast<const float *>(ed)[i] == 0.0f;
    nz += !(zero && ec[i] == 0);
  }
  m->nnz = nz + cnnz;
  m->format_bytes = slots * (vs + 4) + (uint64_t)cnnz * (vs + 8) + (uint64_t)cols * vs + (uint64_t)rows * vs;
  m->ws_bytes = coo_ws_bytes(cnnz);
  unsigned char *ws = nullptr;
  int st;
  if ((st = track_upload_bytes(m, &m->vals, ed, slots * vs)) || (st = track_upload(m, &m->cols_a, ec, slots)) ||
      (st = track_upload_bytes(m, &m->vals2, cd, (size_t)cnnz * vs)) || (st = track_upload(m, &m->cols2, cc, cnnz)) ||
      (st = track_upload(m, &m->rows2, cr, cnnz)) || (st = track(m, &ws, m->ws_bytes))) {
    mfp_matrix_destroy(m);
    return st;
  }
  m->ws = ws;
  if (ws && cudaMemset(ws, 0, m->ws_bytes) != cudaSuccess) {
    mfp_matrix_destroy(m);
    return fail(MFP_ERROR_CUDA, "cudaMemset workspace");
  }
  return finish_matrix(m, out);
}

// Builds a handle from a device CSR: the format's arrays are produced on the
// GPU by the mfp_dev_* converters; only per-plan metadata comes to the host
// (row_ptr for CSR plans, slices_ptr and x windows for SCOO).
int mfp_matrix_create_device(int format, int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp,
                             const uint32_t *ci, const void *data, const mfp_device_build_options *opt,
                             mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (format < 0 || format > MFP_FORMAT_HYBRID || !valid_vt(vt))
    return fail(MFP_ERROR_INVALID_VALUE, "bad format or value type");
  if (nnz && (!ci || !data)) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  int st = mfp_dev_check_csr(rows, cols, nnz, rp, ci, nullptr);
  if (st) return st;
  const mfp_device_build_options o =
      opt ? *opt : mfp_device_build_options{nullptr, MFP_ELL_WIDTH_LONGEST, nullptr, 0u};
  const size_t vs = value_size(vt);
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = format;
  m->value_type = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  auto bail = [&](int status) {
    mfp_matrix_destroy(m);
    return status;
  };
  uint32_t width = o.ell_width;
  if ((format == MFP_FORMAT_ELL || format == MFP_FORMAT_HYBRID) && width == MFP_ELL_WIDTH_LONGEST) {
    mfp_rows_statistic rs{};
    if (rows && (st = mfp_dev_rows_statistics(rows, rp, &rs, nullptr))) return bail(st);
    width = rows ? rs.max_elements_in_rows : 0u;
  }
  const uint64_t xy_bytes = (uint64_t)cols * vs + (uint64_t)rows * vs;
  switch (format) {
    case MFP_FORMAT_CSR_SCALAR:
    case MFP_FORMAT_CSR_VECTOR:
    case MFP_FORMAT_CSR_ADAPTIVE: {
      m->format_bytes = (uint64_t)nnz * (vs + 4) + ((uint64_t)rows + 1) * 4 + xy_bytes;
      std::vector<uint32_t> hrp((size_t)rows + 1);
      if ((st = track_bytes(m, &m->vals, (size_t)nnz * vs)) ||
          (st = track(m, &m->cols_a, nnz)) || (st = track(m, &m->rows_a, (size_t)rows + 1)))
        return bail(st);
      if ((nnz && (cudaMemcpy(m->vals, data, (size_t)nnz * vs, cudaMemcpyDeviceToDevice) != cudaSuccess ||
                   cudaMemcpy(m->cols_a, ci, (size_t)nnz * 4, cudaMemcpyDeviceToDevice) != cudaSuccess)) ||
          cudaMemcpy(m->rows_a, rp, hrp.size() * 4, cudaMemcpyDeviceToDevice) != cudaSuccess ||
          cudaMemcpy(hrp.data(), rp, hrp.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return bail(fail(MFP_ERROR_CUDA, "cudaMemcpy CSR arrays"));
      if ((st = mfp_csr_plan_create(rows, cols, nnz, hrp.data(), format, o.csr, &m->plan))) return bail(st);
      m->device_bytes += m->plan->device_bytes;
      break;
    }
    case MFP_FORMAT_ELL: {
      const uint64_t slots = (uint64_t)rows * width;
      uint32_t dropped = 0;
      if ((st = mfp_dev_coo_count(rows, rp, width, &dropped, nullptr))) return bail(st);
      m->width = width;
      m->nnz = nnz - dropped;
      m->format_bytes = slots * (vs + 4) + xy_bytes;
      if ((st = track_bytes(m, &m->vals, slots * vs)) ||
          (st = track(m, &m->cols_a, slots)) ||
          (st = mfp_dev_ell_from_csr(vt, rows, rp, ci, data, width, m->vals, m->cols_a, nullptr)))
        return bail(st);
      break;
    }
    case MFP_FORMAT_COO:
    case MFP_FORMAT_HYBRID: {
      const bool hyb = format == MFP_FORMAT_HYBRID;
      uint32_t cnnz = nnz;
      if (hyb && (st = mfp_dev_coo_count(rows, rp, width, &cnnz, nullptr))) return bail(st);
      const uint64_t slots = hyb ? (uint64_t)rows * width : 0u;
      void **cv = hyb ? &m->vals2 : &m->vals;
      uint32_t **cc = hyb ? &m->cols2 : &m->cols_a, **cr = hyb ? &m->rows2 : &m->rows_a;
      if (hyb) {
        m->width = width;
        m->coo_nnz = cnnz;
        if ((st = track_bytes(m, &m->vals, slots * vs)) ||
            (st = track(m, &m->cols_a, slots)) ||
            (st = mfp_dev_ell_from_csr(vt, rows, rp, ci, data, width, m->vals, m->cols_a, nullptr)))
          return bail(st);
      }
      m->format_bytes = slots * (vs + 4) + (uint64_t)cnnz * (vs + 8) + xy_bytes;
      m->ws_bytes = coo_ws_bytes(cnnz);
      unsigned char *ws = nullptr;
      if ((st = track_bytes(m, cv, (size_t)cnnz * vs)) || (st = track(m, cc, cnnz)) ||
          (st = track(m, cr, cnnz)) || (st = track(m, &ws, m->ws_bytes)) ||
          (st = mfp_dev_coo_from_csr(vt, rows, rp, ci, data, hyb ? width : 0u, *cv, *cc, *cr, nullptr)))
        return bail(st);
      m->ws = ws;
      if (ws && cudaMemset(ws, 0, m->ws_bytes) != cudaSuccess) return bail(fail(MFP_ERROR_CUDA, "cudaMemset workspace"));
      break;
    }
    case MFP_FORMAT_SCOO: {
      mfp_scoo_params prm{};
      if (o.scoo) {
        prm = *o.scoo;
      } else {
        mfp_device_info di{};
        if ((st = mfp_get_device_info(m->device, &di)) ||
            (st = mfp_scoo_params_compute(rows, di.sm_count, di.shared_mem_per_block, vt, &prm)))
          return bail(st);
      }
      if ((uint64_t)prm.slice_size * prm.slices_count < rows)
        return bail(fail(MFP_ERROR_INVALID_VALUE, "slices do not cover the rows"));
      m->slices = prm.slices_count;
      m->slice_size = prm.slice_size;
      m->format_bytes = (uint64_t)nnz * (vs + 8) + ((uint64_t)m->slices + 1) * 4 + xy_bytes;
      uint32_t *dwin = nullptr;
      if ((st = track_bytes(m, &m->vals, (size_t)nnz * vs)) ||
          (st = track(m, &m->cols_a, nnz)) || (st = track(m, &m->rows_a, nnz)) ||
          (st = track(m, &m->aux, (size_t)m->slices + 1)) || (st = dmalloc(&dwin, 2 * (size_t)m->slices)))
        return bail(st);
      std::vector<uint32_t> win(2 * (size_t)m->slices), hsp((size_t)m->slices + 1);
      st = mfp_dev_scoo_from_csr(vt, rows, nnz, rp, ci, data, &prm, m->vals, m->cols_a, m->rows_a, m->aux, nullptr);
      if (!st && o.scoo_sort_cols && nnz) {
        st = mfp_dev_scoo_sort_cols(vt, rows, cols, prm.slice_size, nnz, m->vals, m->cols_a, m->rows_a, nullptr);
        m->rows_unsorted = true;
      }
      if (!st) st = mfp_dev_scoo_x_windows(nnz, m->cols_a, m->aux, m->slices, dwin, nullptr);
      if (!st && (cudaMemcpy(win.data(), dwin, win.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                  cudaMemcpy(hsp.data(), m->aux, hsp.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess))
        st = fail(MFP_ERROR_CUDA, "cudaMemcpy SCOO metadata");
      cudaFree(dwin);
      if (st || (st = scoo_attach_windows(m, win, hsp.data()))) return bail(st);
      break;
    }
    default:
      return bail(fail(MFP_ERROR_INVALID_VALUE, "bad format"));
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(MFP_ERROR_CUDA, "device conversion"));
  return finish_matrix(m, out);
}

int mfp_matrix_create_lowp(int vt, int index16, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp,
                           const uint32_t *ci, const double *v, mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (nnz && (!ci || !v)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  int st = check_row_ptr(rows, nnz, rp);
  if (st) return st;
  if ((st = check_columns(ci, nnz, cols))) return st;
  std::vector<uint16_t> q(nnz), dl;
  std::vector<float> sc(rows);
  std::vector<uint32_t> bs;
  if ((st = mfp_lowp_quantize(vt, rows, rp, v, q.data(), sc.data()))) return st;
  if (index16) {
    dl.resize(nnz);
    bs.resize(((uint64_t)nnz + MFP_LOWP_DELTA_CHUNK - 1) / MFP_LOWP_DELTA_CHUNK);
    if ((st = mfp_lowp_deltas(nnz, ci, dl.data(), bs.data()))) return st;
  }
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_CSR_LOWP;
  m->value_type = MFP_F32;  // x and y
  m->lowp_vt = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  for (uint32_t r = 0; r < rows && !m->long_rows; ++r) m->long_rows = rp[r + 1] - rp[r] > kLowpTmaMaxRow;
  m->format_bytes = (uint64_t)nnz * (index16 ? 4 : 6) + (uint64_t)bs.size() * 4 + (uint64_t)rows * 4 +
                    ((uint64_t)rows + 1) * 4 + (uint64_t)cols * 4 + (uint64_t)rows * 4;
  if ((st = track_upload(m, &m->rows_a, rp, (size_t)rows + 1)) || (st = track_upload(m, &m->scale, sc.data(), sc.size())) ||
      (st = track_upload_bytes(m, &m->vals, q.data(), q.size() * 2)) ||
      (index16 ? ((st = track_upload(m, &m->delta, dl.data(), dl.size())) ||
                  (st = track_upload(m, &m->base, bs.data(), bs.size())))
               : (st = track_upload(m, &m->cols_a, ci, nnz)))) {
    mfp_matrix_destroy(m);
    return st;
  }
  return finish_matrix(m, out);
}

int mfp_matrix_create_lowp_ell(int vt, int index16, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *rp,
                               const uint32_t *ci, const double *v, mfp_matrix **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (vt != MFP_BF16 && vt != MFP_F16) return fail(MFP_ERROR_INVALID_VALUE, "value type must be BF16 or F16");
  if (nnz && (!ci || !v)) return fail(MFP_ERROR_INVALID_VALUE, "null host array");
  int st = check_row_ptr(rows, nnz, rp);
  if (st) return st;
  if ((st = check_columns(ci, nnz, cols))) return st;
  uint32_t width = 0;
  for (uint32_t r = 0; r < rows; ++r) width = std::max(width, rp[r + 1] - rp[r]);
  const uint64_t slots = (uint64_t)width * rows;
  if (slots > (uint64_t)1 << 33) return fail(MFP_ERROR_TOO_LARGE, "ELL padding: %llu slots", (unsigned long long)slots);
  std::vector<uint16_t> q(slots), off(index16 ? slots : 0);
  std::vector<uint32_t> c32(index16 ? 0 : slots);
  std::vector<float> sc(rows);
  if ((st = mfp_lowp_ell_from_csr(vt, index16, rows, cols, rp, ci, v, width, q.data(),
                                  index16 ? (void *)off.data() : (void *)c32.data(), sc.data())))
    return st;
  auto *m = new mfp_matrix();
  cudaGetDevice(&m->device);
  m->format = MFP_FORMAT_ELL_LOWP;
  m->value_type = MFP_F32;  // x and y
  m->lowp_vt = vt;
  m->rows = rows;
  m->cols = cols;
  m->nnz = nnz;
  m->width = width;
  m->format_bytes = slots * (index16 ? 4 : 6) + (uint64_t)rows * 4 + (uint64_t)cols * 4 + (uint64_t)rows * 4;
  if ((st = track_upload(m, &m->scale, sc.data(), sc.size())) ||
      (st = track_upload_bytes(m, &m->vals, q.data(), q.size() * 2)) ||
      (index16 ? (st = track_upload(m, &m->delta, off.data(), off.size()))
               : (st = track_upload(m, &m->cols_a, c32.data(), c32.size())))) {
    mfp_matrix_destroy(m);
    return st;
  }
  return finish_matrix(m, out);
}

int mfp_matrix_get_info(const mfp_matrix *m, mfp_matrix_info *out) {
  if (!m || !out) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const size_t vs = value_size(m->value_type);
  out->format = m->format;
  const bool lowp = m->format == MFP_FORMAT_CSR_LOWP || m->format == MFP_FORMAT_ELL_LOWP;
  out->value_type = lowp ? m->lowp_vt : m->value_type;
  out->rows = m->rows;
  out->cols = m->cols;
  out->nnz = m->nnz;
  out->format_bytes = m->format_bytes;
  out->algorithmic_bytes = m->nnz * (vs + 4) + ((uint64_t)m->rows + 1) * 4 + (uint64_t)m->cols * vs + (uint64_t)m->rows * vs;
  if (lowp)  // 16-bit values, uint32 column ids, row scales
    out->algorithmic_bytes = m->nnz * 6 + (uint64_t)m->rows * 4 + ((uint64_t)m->rows + 1) * 4 +
                             (uint64_t)m->cols * 4 + (uint64_t)m->rows * 4;
  out->device_bytes = m->device_bytes;
  // the two-pass COO: a warp pass, then the fix-up pass (always for plain COO,
  // which zeroes leading and trailing empty rows there; for the hybrid's
  // accumulating tail only when there is more than one warp tile)
  if (m->format == MFP_FORMAT_COO)
    out->kernel_launches = m->nnz ? 2u : (m->rows ? 1u : 0u);
  else if (m->format == MFP_FORMAT_HYBRID)
    out->kernel_launches = 1u + (m->coo_nnz ? (m->coo_nnz > d::kWarpTile ? 2u : 1u) : 0u);
  else if (m->plan && m->plan->tile)  // CSR vector on short rows: warp pass + fix-up
    out->kernel_launches = 2u;
  else
    out->kernel_launches = 1u;
  return ok();
}

int mfp_matrix_spmv(const mfp_matrix *m, const void *x, void *y, void *stream) {
  if (!m || !y || (!x && m->cols)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const bool f64 = m->value_type == MFP_F64;
  switch (m->format) {
    case MFP_FORMAT_CSR_SCALAR:
    case MFP_FORMAT_CSR_VECTOR:
    case MFP_FORMAT_CSR_ADAPTIVE:
      return f64 ? csr_spmv<double>(m->plan, (const double *)m->vals, m->cols_a, m->rows_a, (const double *)x,
                                    (double *)y, stream)
                 : csr_spmv<float>(m->plan, (const float *)m->vals, m->cols_a, m->rows_a, (const float *)x,
                                   (float *)y, stream);
    case MFP_FORMAT_ELL:
      return f64 ? ell_spmv<double>(m->rows, m->width, (const double *)m->vals, m->cols_a, (const double *)x,
                                    (double *)y, stream)
                 : ell_spmv<float>(m->rows, m->width, (const float *)m->vals, m->cols_a, (const float *)x,
                                   (float *)y, stream);
    case MFP_FORMAT_COO:
      return f64 ? coo_spmv<double>(m->rows, (uint32_t)m->nnz, (const double *)m->vals, m->cols_a, m->rows_a,
                                    (const double *)x, (double *)y, m->ws, m->ws_bytes, stream, m->rel, m->tile_base,
                                    m->rel8, m->wide_tiles > 0)
                 : coo_spmv<float>(m->rows, (uint32_t)m->nnz, (const float *)m->vals, m->cols_a, m->rows_a,
                                   (const float *)x, (float *)y, m->ws, m->ws_bytes, stream, m->rel, m->tile_base,
                                   m->rel8, m->wide_tiles > 0);
    case MFP_FORMAT_SCOO:
      if (m->rows_unsorted)
        return f64 ? scoo_spmv<double, true>(m->rows, m->slices, m->slice_size, (const double *)m->vals, m->cols_a,
                                             m->rows_a, m->aux, m->win, m->max_window, m->order, (const double *)x,
                                             (double *)y, stream)
                   : scoo_spmv<float, true>(m->rows, m->slices, m->slice_size, (const float *)m->vals, m->cols_a,
                                            m->rows_a, m->aux, m->win, m->max_window, m->order, (const float *)x,
                                            (float *)y, stream);
      return f64 ? scoo_spmv<double>(m->rows, m->slices, m->slice_size, (const double *)m->vals, m->cols_a,
                                     m->rows_a, m->aux, m->win, m->max_window, m->order, (const double *)x,
                                     (double *)y, stream, m->rel)
                 : scoo_spmv<float>(m->rows, m->slices, m->slice_size, (const float *)m->vals, m->cols_a, m->rows_a,
                                    m->aux, m->win, m->max_window, m->order, (const float *)x, (float *)y, stream,
                                    m->rel);
    case MFP_FORMAT_HYBRID:
      return f64 ? hyb_spmv<double>(m->rows, m->width, (const double *)m->vals, m->cols_a, m->coo_nnz,
                                    (const double *)m->vals2, m->cols2, m->rows2, (const double *)x, (double *)y,
                                    m->ws, m->ws_bytes, stream, m->rel, m->tile_base, m->rel8, m->wide_tiles > 0)
                 : hyb_spmv<float>(m->rows, m->width, (const float *)m->vals, m->cols_a, m->coo_nnz,
                                   (const float *)m->vals2, m->cols2, m->rows2, (const float *)x, (float *)y, m->ws,
                                   m->ws_bytes, stream, m->rel, m->tile_base, m->rel8, m->wide_tiles > 0);
    case MFP_FORMAT_ELL_LOWP:
      return lowp_ell_spmv(m->lowp_vt, m->rows, m->cols, m->width, (const uint16_t *)m->vals, m->scale,
                           m->delta ? nullptr : m->cols_a, m->delta, (const float *)x, (float *)y, stream);
    case MFP_FORMAT_CSR_LOWP:
      return lowp_spmv(m->lowp_vt, m->rows, (uint32_t)m->nnz, m->rows_a, (const uint16_t *)m->vals, m->scale,
                       m->delta ? nullptr : m->cols_a, m->delta, m->base, (const float *)x, (float *)y, stream,
                       m->long_rows);
    default:
      return fail(MFP_ERROR_INVALID_VALUE, "unknown format %d", m->format);
  }
}

// Formats whose kernels write each row of y once, a warp's stores covering
// consecutive rows: their y can go straight into a page-locked host buffer.
static bool writes_y_in_row_order(const mfp_matrix *m) {
  if (m->plan && (m->plan->cfg.kernel == 2 || m->plan->cfg.kernel == 3)) return false;  // streaming CSR
  switch (m->format) {
    case MFP_FORMAT_CSR_SCALAR:
    case MFP_FORMAT_CSR_ADAPTIVE:
    case MFP_FORMAT_ELL:
    case MFP_FORMAT_SCOO:
    case MFP_FORMAT_CSR_LOWP:
    case MFP_FORMAT_ELL_LOWP:
      return !(m->plan && m->plan->tile) && !m->rows_unsorted;
    case MFP_FORMAT_CSR_VECTOR:
      return !(m->plan && m->plan->tile);
    default:  // COO and the warp-tile kernels write rows as their tiles finish; the hybrid adds into y
      return false;
  }
}

int mfp_matrix_spmv_host(mfp_matrix *m, const void *hx, void *hy, void *stream) {
  if (!m || !hy || (!hx && m->cols)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const size_t vs = value_size(m->value_type);
  cudaStream_t s = as_stream(stream);
  // a page-locked y (cudaHostAlloc / cudaHostRegister) that the device can
  // address takes the kernel's stores directly, so the copy-out overlaps the
  // kernel instead of following it
  void *y_mapped = nullptr;
  if (m->rows && writes_y_in_row_order(m)) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, hy) == cudaSuccess && a.type == cudaMemoryTypeHost && a.devicePointer)
      y_mapped = a.devicePointer;
    else
      cudaGetLastError();
  }
  if (m->cols)
    CUDA_TRY(cudaMemcpyAsync(m->dx, hx, (size_t)m->cols * vs, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync x");
  int st = mfp_matrix_spmv(m, m->dx, y_mapped ? y_mapped : m->dy, stream);
  if (st) return st;
  if (m->rows && !y_mapped)
    CUDA_TRY(cudaMemcpyAsync(hy, m->dy, (size_t)m->rows * vs, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync y");
  CUDA_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return ok();
}

int mfp_matrix_spmv_host_batch(mfp_matrix *m, uint32_t count, const void *const *hx, void *const *hy,
                               void *stream) {
  if (!m || (count && (!hx || !hy))) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  for (uint32_t i = 0; i < count; ++i)
    if (!hy[i] || (!hx[i] && m->cols)) return fail(MFP_ERROR_INVALID_VALUE, "null host vector %u", i);
  if (count == 0) return ok();
  const size_t vs = value_size(m->value_type);
  cudaStream_t s = as_stream(stream);
  if (!m->s_in) {
    unsigned char *a = nullptr, *b = nullptr;
    int st = track(m, &a, (size_t)std::max(1u, m->cols) * vs);
    if (!st) st = track(m, &b, (size_t)std::max(1u, m->rows) * vs);
    if (st) return st;
    m->dx2 = a;
    m->dy2 = b;
    for (cudaEvent_t *e : {&m->ev_start, &m->ev_in[0], &m->ev_in[1], &m->ev_k[0], &m->ev_k[1], &m->ev_out[0],
                           &m->ev_out[1]})
      CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "cudaEventCreateWithFlags");
    CUDA_TRY(cudaStreamCreateWithFlags(&m->s_out, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    CUDA_TRY(cudaStreamCreateWithFlags(&m->s_in, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
  }
  void *dx[2] = {m->dx, m->dx2}, *dy[2] = {m->dy, m->dy2};
  // the copies start after the work already on `stream`
  CUDA_TRY(cudaEventRecord(m->ev_start, s), "cudaEventRecord");
  CUDA_TRY(cudaStreamWaitEvent(m->s_in, m->ev_start, 0), "cudaStreamWaitEvent");
  CUDA_TRY(cudaStreamWaitEvent(m->s_out, m->ev_start, 0), "cudaStreamWaitEvent");
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t b = i & 1u;
    // x_i into staging b once SpMV i - 2 has read it
    if (i >= 2) CUDA_TRY(cudaStreamWaitEvent(m->s_in, m->ev_k[b], 0), "cudaStreamWaitEvent");
    if (m->cols)
      CUDA_TRY(cudaMemcpyAsync(dx[b], hx[i], (size_t)m->cols * vs, cudaMemcpyHostToDevice, m->s_in),
               "cudaMemcpyAsync x");
    CUDA_TRY(cudaEventRecord(m->ev_in[b], m->s_in), "cudaEventRecord");
    // SpMV i once x_i is in and y_{i-2} is out of staging b
    CUDA_TRY(cudaStreamWaitEvent(s, m->ev_in[b], 0), "cudaStreamWaitEvent");
    if (i >= 2) CUDA_TRY(cudaStreamWaitEvent(s, m->ev_out[b], 0), "cudaStreamWaitEvent");
    const int st = mfp_matrix_spmv(m, dx[b], dy[b], stream);
    if (st) {
      cudaStreamSynchronize(m->s_in);
      cudaStreamSynchronize(m->s_out);
      return st;
    }
    CUDA_TRY(cudaEventRecord(m->ev_k[b], s), "cudaEventRecord");
    CUDA_TRY(cudaStreamWaitEvent(m->s_out, m->ev_k[b], 0), "cudaStreamWaitEvent");
    if (m->rows)
      CUDA_TRY(cudaMemcpyAsync(hy[i], dy[b], (size_t)m->rows * vs, cudaMemcpyDeviceToHost, m->s_out),
               "cudaMemcpyAsync y");
    CUDA_TRY(cudaEventRecord(m->ev_out[b], m->s_out), "cudaEventRecord");
  }
  // `stream` ends after the last copy-out (copies are ordered on s_out)
  CUDA_TRY(cudaStreamWaitEvent(s, m->ev_out[(count - 1u) & 1u], 0), "cudaStreamWaitEvent");
  CUDA_TRY(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return ok();
}

int mfp_matrix_time(const mfp_matrix *m, const void *x, void *y, uint32_t reps, int flush_l2, void *stream,
                    double *mean_s, double *median_s) {
  if (!m || reps == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  cudaStream_t s = as_stream(stream);
  static void *flush_buf = nullptr;
  static size_t flush_bytes = 0;
  static std::mutex mu;
  if (flush_l2) {
    std::lock_guard<std::mutex> g(mu);
    if (!flush_buf) {
      int dev = 0;
      cudaGetDevice(&dev);
      int l2 = 0;
      cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
      flush_bytes = (size_t)std::max(l2, 1 << 20) * 2;
      CUDA_TRY(cudaMalloc(&flush_buf, flush_bytes), "cudaMalloc flush buffer");
    }
  }
  std::vector<cudaEvent_t> ev(2 * (size_t)reps);
  for (auto &e : ev) CUDA_TRY(cudaEventCreate(&e), "cudaEventCreate");
  int st = MFP_SUCCESS;
  for (uint32_t i = 0; i < reps && !st; ++i) {
    if (flush_l2) cudaMemsetAsync(flush_buf, (int)(i & 0xff), flush_bytes, s);
    cudaEventRecord(ev[2 * i], s);
    st = mfp_matrix_spmv(m, x, y, stream);
    cudaEventRecord(ev[2 * i + 1], s);
  }
  std::vector<double> t;
  if (!st) {
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_fail(e, "cudaStreamSynchronize");
  }
  if (!st)
    for (uint32_t i = 0; i < reps; ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      t.push_back(ms * 1e-3);
    }
  for (auto &e : ev) cudaEventDestroy(e);
  if (st) return st;
  double sum = 0;
  for (double v : t) sum += v;
  std::sort(t.begin(), t.end());
  if (mean_s) *mean_s = sum / reps;
  if (median_s) *median_s = t[t.size() / 2];
  return ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Format selector network (engine extension)
// ---------------------------------------------------------------------------
extern "C" {

uint32_t mfp_mlp_param_count(void) { return d::kMlpParams; }

int mfp_mlp_forward(const float *P, const float *x, uint32_t B, float *h1, float *h2, float *y, void *stream) {
  if (B == 0) return ok();
  if (!P || !x || !h1 || !h2 || !y) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  cudaStream_t s = as_stream(stream);
  auto grid = [](uint64_t n) { return (uint32_t)((n + 255) / 256); };
  d::mlp_dense_fwd<true><<<grid((uint64_t)B * d::kMlpHid), 256, 0, s>>>(x, P + d::kMlpW1, P + d::kMlpB1, h1, B,
                                                                       d::kMlpIn, d::kMlpHid);
  d::mlp_dense_fwd<true><<<grid((uint64_t)B * d::kMlpHid), 256, 0, s>>>(h1, P + d::kMlpW2, P + d::kMlpB2, h2, B,
                                                                       d::kMlpHid, d::kMlpHid);
  d::mlp_dense_fwd<false><<<grid((uint64_t)B * d::kMlpOut), 256, 0, s>>>(h2, P + d::kMlpW3, P + d::kMlpB3, y, B,
                                                                        d::kMlpHid, d::kMlpOut);
  return check_launch("mlp forward");
}

int mfp_mlp_backward(const float *P, const float *x, const float *h1, const float *h2, const float *y,
                     const float *t, const float *mask, uint32_t B, float *G, float *loss, float *work,
                     void *stream) {
  if (!P || !G || !loss || (B && (!x || !h1 || !h2 || !y || !t || !mask || !work)))
    return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  cudaStream_t s = as_stream(stream);
  if (B == 0) {
    CUDA_TRY(cudaMemsetAsync(G, 0, d::kMlpParams * sizeof(float), s), "cudaMemsetAsync");
    CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(float), s), "cudaMemsetAsync");
    return ok();
  }
  float *dY = work, *dZ2 = work + (size_t)B * d::kMlpOut, *dZ1 = dZ2 + (size_t)B * d::kMlpHid;
  auto grid = [](uint64_t n) { return (uint32_t)((n + 255) / 256); };
  d::mlp_loss_grad<<<1, 1024, 0, s>>>(y, t, mask, B * d::kMlpOut, dY, loss);
  d::mlp_dense_bwd_w<<<grid(d::kMlpHid * d::kMlpOut + d::kMlpOut), 256, 0, s>>>(h2, dY, G + d::kMlpW3, G + d::kMlpB3,
                                                                                B, d::kMlpHid, d::kMlpOut);
  d::mlp_dense_bwd_in<<<grid((uint64_t)B * d::kMlpHid), 256, 0, s>>>(dY, P + d::kMlpW3, h2, dZ2, B, d::kMlpHid,
                                                                      d::kMlpOut);
  d::mlp_dense_bwd_w<<<grid(d::kMlpHid * d::kMlpHid + d::kMlpHid), 256, 0, s>>>(h1, dZ2, G + d::kMlpW2,
                                                                                G + d::kMlpB2, B, d::kMlpHid,
                                                                                d::kMlpHid);
  d::mlp_dense_bwd_in<<<grid((uint64_t)B * d::kMlpHid), 256, 0, s>>>(dZ2, P + d::kMlpW2, h1, dZ1, B, d::kMlpHid,
                                                                      d::kMlpHid);
  d::mlp_dense_bwd_w<<<grid(d::kMlpIn * d::kMlpHid + d::kMlpHid), 256, 0, s>>>(x, dZ1, G + d::kMlpW1, G + d::kMlpB1,
                                                                               B, d::kMlpIn, d::kMlpHid);
  return check_launch("mlp backward");
}

int mfp_mlp_adam(float *p, const float *g, float *m, float *v, uint32_t n, float lr, float beta1, float beta2,
                 float eps, uint32_t step, void *stream) {
  if (n == 0) return ok();
  if (!p || !g || !m || !v || step == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  const float c1 = 1.f - (float)std::pow((double)beta1, (double)step);
  const float c2 = 1.f - (float)std::pow((double)beta2, (double)step);
  d::mlp_adam<<<(n + 255) / 256, 256, 0, as_stream(stream)>>>(p, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return check_launch("mlp adam");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched SpMV: many matrices as one block-diagonal CSR (engine extension)
// ---------------------------------------------------------------------------
struct mfp_batch {
  int device = 0, vt = 0;
  uint32_t n = 0, rows = 0, cols = 0, nnz = 0;
  std::vector<uint64_t> x_off, y_off;
  std::vector<uint32_t> host_rp;  // concatenated row_ptr (for re-planning)
  uint64_t algorithmic_bytes = 0;
  void *vals = nullptr;
  uint32_t *cols_a = nullptr, *rp = nullptr;
  size_t array_bytes = 0;
  mfp_csr_plan *plan = nullptr;
  mfp_batch_config cfg{};
  // captured graph of one launch for (gx, gy)
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *gx = nullptr;
  void *gy = nullptr;
};

namespace {
void batch_drop_graph(mfp_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->gx = nullptr;
  b->gy = nullptr;
}
int batch_plan(mfp_batch *b, const mfp_batch_config &c, mfp_csr_plan **out) {
  if (c.algo < 0 || c.algo > 2) return fail(MFP_ERROR_INVALID_VALUE, "batch algo must be 0, 1 or 2");
  return mfp_csr_plan_create(b->rows, b->cols, b->nnz, b->host_rp.data(), c.algo, &c.csr, out);
}
int batch_launch(const mfp_batch *b, const mfp_csr_plan *plan, const void *x, void *y, void *stream) {
  return b->vt == MFP_F64 ? csr_spmv<double>(plan, (const double *)b->vals, b->cols_a, b->rp, (const double *)x,
                                             (double *)y, stream)
                          : csr_spmv<float>(plan, (const float *)b->vals, b->cols_a, b->rp, (const float *)x,
                                            (float *)y, stream);
}
}  // namespace

extern "C" {

int mfp_batch_create(int vt, uint32_t n, const uint32_t *rows, const uint32_t *cols, const uint32_t *const *row_ptr,
                     const uint32_t *const *columns, const void *const *values, mfp_batch **out) {
  if (!out) return fail(MFP_ERROR_INVALID_VALUE, "null output");
  *out = nullptr;
  if (!valid_vt(vt)) return fail(MFP_ERROR_INVALID_VALUE, "bad value type");
  if (n && (!rows || !cols || !row_ptr || !columns || !values)) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  const size_t vs = value_size(vt);
  auto b = std::make_unique<mfp_batch>();
  cudaGetDevice(&b->device);
  b->vt = vt;
  b->n = n;
  b->x_off.assign((size_t)n + 1, 0);
  b->y_off.assign((size_t)n + 1, 0);
  uint64_t R = 0, Cn = 0, Z = 0;
  for (uint32_t k = 0; k < n; ++k) {
    if (!row_ptr[k]) return fail(MFP_ERROR_INVALID_VALUE, "null row_ptr of matrix %u", k);
    const uint32_t nz = row_ptr[k][rows[k]];
    int st = check_row_ptr(rows[k], nz, row_ptr[k]);
    if (!st && nz && (!columns[k] || !values[k])) st = fail(MFP_ERROR_INVALID_VALUE, "null arrays");
    if (!st) st = check_columns(columns[k], nz, cols[k]);
    if (st) {
      const std::string msg = mfp_last_error();
      return fail(st, "matrix %u: %s", k, msg.c_str());
    }
    b->x_off[k] = Cn;
    b->y_off[k] = R;
    R += rows[k];
    Cn += cols[k];
    Z += nz;
    b->algorithmic_bytes += (uint64_t)nz * (vs + 4) + ((uint64_t)rows[k] + 1) * 4 + (uint64_t)cols[k] * vs +
                            (uint64_t)rows[k] * vs;
  }
  b->x_off[n] = Cn;
  b->y_off[n] = R;
  if (R >= UINT32_MAX || Cn >= UINT32_MAX || Z >= UINT32_MAX)
    return fail(MFP_ERROR_TOO_LARGE, "batch totals exceed 32-bit indexing (rows %llu, cols %llu, nnz %llu)",
                (unsigned long long)R, (unsigned long long)Cn, (unsigned long long)Z);
  b->rows = (uint32_t)R;
  b->cols = (uint32_t)Cn;
  b->nnz = (uint32_t)Z;
  b->host_rp.resize((size_t)R + 1);
  std::vector<uint32_t> hc(Z);
  std::vector<unsigned char> hv(Z * vs);
  uint64_t r0 = 0, z0 = 0;
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t nz = row_ptr[k][rows[k]];
    for (uint32_t r = 0; r < rows[k]; ++r) b->host_rp[r0 + r] = (uint32_t)(z0 + row_ptr[k][r]);
    const uint32_t xo = (uint32_t)b->x_off[k];
    for (uint32_t e = 0; e < nz; ++e) hc[z0 + e] = columns[k][e] + xo;
    if (nz) std::memcpy(hv.data() + z0 * vs, values[k], (size_t)nz * vs);
    r0 += rows[k];
    z0 += nz;
  }
  b->host_rp[R] = (uint32_t)Z;
  unsigned char *dv = nullptr;
  int st;
  if ((st = dmalloc(&dv, hv.size(), &b->array_bytes)) || (st = dmalloc(&b->cols_a, hc.size(), &b->array_bytes)) ||
      (st = dmalloc(&b->rp, b->host_rp.size(), &b->array_bytes))) {
    cudaFree(dv);
    mfp_batch_destroy(b.release());
    return st;
  }
  b->vals = dv;
  if ((!hv.empty() && cudaMemcpy(dv, hv.data(), hv.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
      (!hc.empty() && cudaMemcpy(b->cols_a, hc.data(), hc.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(b->rp, b->host_rp.data(), b->host_rp.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    mfp_batch_destroy(b.release());
    return fail(MFP_ERROR_CUDA, "batch upload failed");
  }
  b->cfg = mfp_batch_config{};
  if ((st = batch_plan(b.get(), b->cfg, &b->plan))) {
    mfp_batch_destroy(b.release());
    return st;
  }
  *out = b.release();
  return ok();
}

int mfp_batch_destroy(mfp_batch *b) {
  if (!b) return ok();
  batch_drop_graph(b);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  mfp_csr_plan_destroy(b->plan);
  cudaFree(b->vals);
  cudaFree(b->cols_a);
  cudaFree(b->rp);
  delete b;
  return ok();
}

int mfp_batch_offsets(const mfp_batch *b, uint64_t *xo, uint64_t *yo) {
  if (!b) return fail(MFP_ERROR_INVALID_VALUE, "null batch");
  if (xo) std::copy(b->x_off.begin(), b->x_off.end(), xo);
  if (yo) std::copy(b->y_off.begin(), b->y_off.end(), yo);
  return ok();
}

int mfp_batch_get_info(const mfp_batch *b, mfp_batch_info *out) {
  if (!b || !out) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  out->matrices = b->n;
  out->rows = b->rows;
  out->cols = b->cols;
  out->nnz = b->nnz;
  out->algorithmic_bytes = b->algorithmic_bytes;
  out->device_bytes = b->array_bytes + (b->plan ? b->plan->device_bytes : 0);
  out->config = b->cfg;
  out->kernel_launches = b->nnz ? 1 : (b->rows ? 1 : 0);
  return ok();
}

int mfp_batch_set_config(mfp_batch *b, const mfp_batch_config *c) {
  if (!b || !c) return fail(MFP_ERROR_INVALID_VALUE, "null argument");
  mfp_csr_plan *p = nullptr;
  int st = batch_plan(b, *c, &p);
  if (st) return st;
  batch_drop_graph(b);
  mfp_csr_plan_destroy(b->plan);
  b->plan = p;
  b->cfg = *c;
  return ok();
}

int mfp_batch_spmv(const mfp_batch *b, const void *x, void *y, void *stream) {
  if (!b) return fail(MFP_ERROR_INVALID_VALUE, "null batch");
  return batch_launch(b, b->plan, x, y, stream);
}

int mfp_batch_autotune(mfp_batch *b, const void *x, void *y, uint32_t reps, void *stream, mfp_batch_config *chosen,
                       double *best_seconds) {
  if (!b || reps == 0) return fail(MFP_ERROR_INVALID_VALUE, "bad argument");
  // the candidate plans: CSR scalar with several warp-assist and long-row
  // thresholds, the streaming (persistent) kernel, CSR vector lane counts and
  // CSR-Adaptive bin sizes
  std::vector<mfp_batch_config> cand;
  auto add = [&](int algo, uint32_t lanes, uint32_t bin, uint32_t assist, uint32_t longt, uint32_t kernel) {
    mfp_batch_config c{};
    c.algo = algo;
    c.csr.vector_lanes = lanes;
    c.csr.bin_nnz = bin;
    c.csr.assist_threshold = assist;
    c.csr.long_row_threshold = longt;
    c.csr.kernel = kernel;
    cand.push_back(c);
  };
  for (uint32_t assist : {32u, 64u, 256u})
    for (uint32_t longt : {2048u, 4096u, 16384u}) add(0, 0, 0, assist, longt, 1);
  add(0, 0, 0, 0, 0, 2);
  add(0, 0, 0, 0, 0, 3);
  for (uint32_t lanes : {0u, 4u, 8u, 32u}) add(1, lanes, 0, 0, 0, 1);
  for (uint32_t bin : {0u, 1020u, 508u}) add(2, 0, bin, 0, 0, 1);
  cudaStream_t s = as_stream(stream);
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0), "cudaEventCreate");
  CUDA_TRY(cudaEventCreate(&e1), "cudaEventCreate");
  double best = 1e300;
  int best_i = -1, st = MFP_SUCCESS;
  for (size_t i = 0; i < cand.size() && !st; ++i) {
    mfp_csr_plan *p = nullptr;
    if (batch_plan(b, cand[i], &p)) continue;  // a configuration the matrix does not admit
    std::vector<double> t;
    st = batch_launch(b, p, x, y, stream);  // warm-up
    for (uint32_t r = 0; r < reps && !st; ++r) {
      cudaEventRecord(e0, s);
      st = batch_launch(b, p, x, y, stream);
      cudaEventRecord(e1, s);
      if (!st) {
        const cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaEventSynchronize");
      }
      float ms = 0;
      if (!st) cudaEventElapsedTime(&ms, e0, e1);
      t.push_back(ms * 1e-3);
    }
    mfp_csr_plan_destroy(p);
    if (st) break;
    std::sort(t.begin(), t.end());
    const double med = t[t.size() / 2];
    if (med < best) {
      best = med;
      best_i = (int)i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  if (best_i < 0) return fail(MFP_ERROR_NOT_SUPPORTED, "no candidate plan could be built");
  if ((st = mfp_batch_set_config(b, &cand[best_i]))) return st;
  if (chosen) *chosen = cand[best_i];
  if (best_seconds) *best_seconds = best;
  return ok();
}

int mfp_batch_graph_launch(mfp_batch *b, const void *x, void *y, void *stream) {
  if (!b) return fail(MFP_ERROR_INVALID_VALUE, "null batch");
  if (!b->exec || b->gx != x || b->gy != y) {
    batch_drop_graph(b);
    if (!b->cap_stream) CUDA_TRY(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    CUDA_TRY(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    const int st = batch_launch(b, b->plan, x, y, b->cap_stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap_stream, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&b->exec, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) {
      b->exec = nullptr;
      return cuda_fail(e2, "cudaGraphInstantiate");
    }
    b->gx = x;
    b->gy = y;
  }
  CUDA_TRY(cudaGraphLaunch(b->exec, as_stream(stream)), "cudaGraphLaunch");
  return ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// COO SpMV that allocates nothing (no counterpart in the reference)
// ---------------------------------------------------------------------------
// Some callers cannot let a library call cudaMalloc: hosts that hand out all
// device memory through their own pool or budget, and loops that cannot
// afford cudaMalloc's latency and implicit synchronisation.  This entry point
// runs the same two-pass COO as mfp_coo_spmv_f32 and keeps its workspace (the
// per-warp-tile partial sums) in a fixed array that is part of the library
// image instead.  The two passes have no waits, so there is no error state to
// report after the launch; the workspace needs no clearing, since every call
// rewrites what it reads.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB on every device that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
void *g_noalloc_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (host code cannot
// use the array's name as an address).  Resolved once per device.
int noalloc_scratch(void **out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(MFP_ERROR_NOT_SUPPORTED, "device %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return MFP_SUCCESS;
}
}  // namespace

extern "C" int mfp_coo_spmv_f32_noalloc(uint32_t rows, uint32_t cols, uint32_t nnz, const float *data,
                                        const uint32_t *col_ids, const uint32_t *row_ids, const float *x, float *y,
                                        void *stream) {
  (void)cols;
  const size_t need = coo_ws_bytes(nnz);
  if (need > kNoAllocScratchBytes)
    return fail(MFP_ERROR_TOO_LARGE,
                "nnz %u needs %zu bytes of COO scratch; the fixed scratch holds %zu bytes (nnz <= %zu)", nnz, need,
                kNoAllocScratchBytes, (kNoAllocScratchBytes - sizeof(d::coo_ws_header)) / 24u * d::kWarpTile);
  if (rows == 0) return ok();
  if (!y) return fail(MFP_ERROR_INVALID_VALUE, "null y");
  if (nnz && (!data || !col_ids || !row_ids || !x)) return fail(MFP_ERROR_INVALID_VALUE, "null device array");
  void *ws = nullptr;
  const int st = noalloc_scratch(&ws);
  if (st) return st;
  return coo_spmv<float>(rows, nnz, data, col_ids, row_ids, x, y, ws, need, stream);
}
