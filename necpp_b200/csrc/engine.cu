// necgpu engine: device buffers, kernel orchestration and the C-ABI of
// include/necgpu.h.  One engine per nec_context; all work goes to one
// stream.  There is no CPU fallback: every compute step is a kernel.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <cstring>
#include <mutex>
#include <atomic>
#include <thread>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/necgpu.h"
#include "fill.cuh"
#include "gemm_tc.cuh"
#include "gemm_dmma.cuh"
#include "lu.cuh"
#include "pattern.cuh"
#include "solve.cuh"
#include "batch.cuh"
#include "somm.cuh"
#include "nearfield.cuh"
#include "peak.cuh"

using namespace necb;

namespace {
constexpr int kNB = 64;  // LU panel width
}

// What the launch sequence of a block-pivoted LU depends on: its size, its
// tuning, its kernels' switches and every buffer and stream it names.
struct LuGraphKey {
  int64_t n = 0, ld = 0, outer = 0;
  int la = 0, la_sms = 0, group = 0, use_tc = 0, trsm8 = 0, nsm = 0;
  const void* ptr[16] = {};
  bool operator==(const LuGraphKey& o) const {
    if (n != o.n || ld != o.ld || outer != o.outer || la != o.la || la_sms != o.la_sms || group != o.group ||
        use_tc != o.use_tc || trsm8 != o.trsm8 || nsm != o.nsm)
      return false;
    for (int i = 0; i < 16; i++)
      if (ptr[i] != o.ptr[i]) return false;
    return true;
  }
};

struct necgpu_engine {
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  int64_t n = 0, ld = 0;
  int64_t launches = 0;
  bool timing = false;
  necgpu_stats stats{};

  FieldParams P{};
  int ground = 0, use_exk = 0;
  double* d_seg = nullptr;  // 8n: x y z s b cab sab salp
  int32_t* d_ind = nullptr; // 2n
  int32_t *d_tile_ptr = nullptr, *d_tsrc = nullptr, *d_tsrc_eptr = nullptr;
  uint8_t* d_ecol = nullptr;
  double* d_ecoef = nullptr;  // 3*ne
  int64_t ne = 0;
  int ntiles = 0;
  int32_t *d_cptr = nullptr, *d_cbasis = nullptr;
  double* d_ccoef = nullptr;
  int64_t nc = 0;

  double2* Z64 = nullptr;
  float2* Z32 = nullptr;
  int factored = -1;  // precision of the factors held, -1 none
  // a setting was changed or a test or batch entry point used since the
  // engine was created: necgpu_release destroys it instead of pooling it
  bool touched = false;
  bool filled = false;
  int* d_piv = nullptr;
  int* d_src = nullptr;  // block-pivoted LU: gather order of each diagonal block's rows
  int* d_perm = nullptr;

  double* d_cand_val = nullptr;
  float* d_cand_valf = nullptr;
  int* d_cand_row = nullptr;
  double2* d_cand_rows = nullptr;  // sized for FP64 (also used as float2)
  double2* d_rowc = nullptr;
  unsigned* d_counter = nullptr;
  int* d_status = nullptr;  // [4]

  double2 *d_b = nullptr, *d_x = nullptr, *d_r = nullptr, *d_cur = nullptr;
  double2 *d_w1 = nullptr, *d_w2 = nullptr;  // factor-precision work (sized FP64)
  double* d_abc = nullptr;
  double* d_rn2 = nullptr;
  int pat_cap = 0;
  double *d_theta = nullptr, *d_phi = nullptr;
  double2 *d_eth = nullptr, *d_eph = nullptr;
  int res_ndir = 0;  // resident pattern directions (bench)
  bool res_rhs = false;

  double refine_tol = 1e-13;
  int refine_max = 30;
  bool have_solution = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int timing_level = 0;
  // per-launch kernel timing (level 2): event pairs pending until a sync
  struct PendingK {
    int cls, ev;
    double flops;
    int stream;        // 0 engine stream, 2 / 3 / 4 the far update, U12 and bulk L21 streams, 1 other
    const char* name;  // launch expression (static storage) or null
  };
  // timing level 3: every timed launch with its start and end on a common
  // time origin (necgpu_get_trace)
  cudaEvent_t trace_base = nullptr;
  bool trace_based = false;
  std::vector<necgpu_trace_rec> trace;
  std::vector<cudaEvent_t> kev;
  int kev_used = 0;
  std::vector<PendingK> kpend;
  int last_ndir = 0;     // directions of the last necgpu_pattern call
  bool last_rhs = false; // d_b holds the last right-hand side
  // triangular solves: persistent sweeps (flags per 64-row block, epoch per sweep)
  bool sweep_trsv = true;
  int* d_flags = nullptr;
  int flag_epoch = 0;
  // tensor-core trailing update of the FP32 LU: packed operands (raw bytes,
  // in the format of the factorisation: gemm_tc.cuh's SplitBf16 or Tf32)
  bool use_tc = true;
  unsigned char *d_Ap = nullptr, *d_Bp = nullptr;
  int64_t tc_rows = 0;
  int64_t tc_kbytes = 0;  // bytes per operand row
  // second packed-operand set (the lookahead's far update)
  unsigned char *d_Ap2 = nullptr, *d_Bp2 = nullptr;
  int64_t tc_rows2 = 0;
  int64_t tc_kbytes2 = 0;
  unsigned tc_attr = 0;  // formats whose GEMM kernel has its shared-memory size set
  // operand format of the mixed LU's update: 0 chooses (TF32 from
  // tf32_min_n unknowns on, split BF16 below that or once a TF32
  // factorisation needed more than tf32_max_iters refinement steps), 1 split
  // BF16, 2 TF32; tc_format_used: the held factors' format
  int tc_format = 0;
  int tc_format_used = 0;
  int64_t tf32_min_n = 10240;
  int tf32_max_iters = 5;
  bool tf32_demoted = false;
  // lookahead: the trailing update beyond the next outer block runs on
  // stream2 with lookahead_sms SMs left free for the next panel
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_far = nullptr;
  // stream3: each inner panel's U12 solve beside its L21 solve
  cudaStream_t stream3 = nullptr;
  // stream4: each inner panel's L21 solve and update below the next
  // panel's rows, beside the next diagonal LU; its B operand alternates
  // between d_Bp and d_Bp3
  cudaStream_t stream4 = nullptr;
  cudaEvent_t ev_diag = nullptr, ev_bulk = nullptr;
  unsigned char* d_Bp3 = nullptr;
  size_t bp3_bytes = 0;
  bool inner_split = true;
  // the split path's next-block rows (L21, U12 and their update) in one
  // launch (panel_top_kernel), the panel's interchanges on stream3
  bool panel_top = true;
  // refinement sweeps in thread-block clusters of this many CTAs (16 or 8;
  // 0: none), with the solved blocks handed over in shared memory
  int sweep_cluster = 16;
  unsigned* d_top_cnt = nullptr;  // panel_top_kernel's arrival counters (zero between launches)
  unsigned char* d_Bpan = nullptr;  // its B operand slots, one per panel of an outer block
  size_t bpan_bytes = 0;
  // L21 rows left-looking with a CTA per 32 rows (l21_rows_kernel) instead
  // of one row per thread
  bool l21_rows = true;
  // CTAs of the rows-below-the-block work on stream4 (L21 solve and update)
  int side_ctas = 32;
  cudaEvent_t ev_swap = nullptr;
  // launch priority of the panel chain's kernels (0: the streams' own)
  int chain_prio = 0;
  cudaEvent_t ev_u12a = nullptr, ev_u12b = nullptr;
  // tuning in effect for the current factorisation (select_tuning)
  bool lookahead = true;
  int lookahead_sms = 48;
  // m-tiles per band of the tensor-core update's tile walk
  int gemm_group = 16;
  bool matrix_only = false;      // necgpu_matrix_solve: a caller's matrix, no structure tables
  // the fill also writes the complex64 copy the mixed LU factors (skipping
  // the demotion pass) when the next factorisation is announced as mixed
  int fill_precision = -1;
  bool z32_fresh = false;  // Z32 holds the demoted current Z64
  // CUDA graph of the block-pivoted LU's launches (run_lu_blockpiv)
  bool lu_graphs = true;
  bool u12_fused = true;  // the outer row block's U12 in one launch
  bool fused_pack = true;  // inner panel solves write the update's packed operands
  LuGraphKey lu_seen{}, lu_key{};
  cudaGraphExec_t lu_exec = nullptr;
  int64_t lu_exec_launches = 0;
  bool tuning_explicit = false;  // necgpu_set_tuning
  necgpu_tuning tuning_set{};
  // environment overrides read at creation (0 / -1: not given)
  int env_outer = 0, env_lookahead_sms = 0, env_lookahead = -1, env_group = 0;
  bool trsm8 = true;  // U12 panel solves with eight warps per vector block (else one thread per vector)
  CUtensorMap tmA{}, tmB{};
  float2* d_dinv = nullptr;  // reciprocal diagonal of U (block-pivoted mixed LU)
  double2* d_zload = nullptr;  // impedance loading per segment (null: unloaded)
  // Sommerfeld ground: tables of the current frequency, the interpolation
  // cache the next fill starts from (kept across fills, as the reference's
  // ground object keeps it), and the near-pair fields of the last fill
  cplx* d_somm = nullptr;
  bool somm_ready = false;
  InterpKey interp_key{kInterpFresh, 0, 0, 0};
  InterpCache* d_interp_carry = nullptr;  // the cache interp_key (carry = 1) stands for
  cplx* d_near_g = nullptr;
  int64_t near_g_cap = 0;
  InterpKey* d_near_entry = nullptr;
  NearRecord* d_near_rec = nullptr;
  int* d_near_cols = nullptr;
  int64_t near_cap = 0;
  float2* d_tinv = nullptr;  // inverted 64 x 64 diagonal blocks of the complex64 factors
  float2* d_wnext = nullptr;  // their products with the neighbouring tile (next_tile_kernel)
  float2* d_wnextT = nullptr;  // the same for the transposed factors (adjoint solves)
  // adjoint solves: transposed factors, matrix and block inverses
  float2* ZT32 = nullptr;
  double2* ZT64 = nullptr;
  float2* d_tinvT = nullptr;
  bool adj_ready = false;
  double2 *d_adj_phi = nullptr, *d_adj_w = nullptr, *d_adj_r = nullptr;
  int adj_cap = 0;  // right-hand sides the adjoint buffers hold
  // perturbed structures (adjoint gradients)
  double *d_pseg = nullptr, *d_pecoef = nullptr, *d_pccoef = nullptr, *d_pout = nullptr;
  double2 *d_pw = nullptr, *d_pfar = nullptr;
  FillArgs* d_pargs = nullptr;
  ContractArgs* d_pcargs = nullptr;
  int p_cap = 0, pw_cap = 0;
  double2* d_pwts = nullptr;  // far-field weights (2 n)
  // host copies of the basis-table layout and end flags (adjoint gradients)
  std::vector<int32_t> h_tptr, h_tbasis, h_ind;
  unsigned* d_sweep_ctr = nullptr;  // progress of the refinement sweeps
  bool inv_sweep = true;
  bool use_dmma = true;  // FP64 trailing update on the FP64 tensor cores
  int64_t outer = 256;  // outer block of the block-pivoted mixed LU (multiple of 64)
  // mixed path: block-local pivoting first, full partial pivoting as fallback
  bool prefer_blockpiv = true;
  bool blockpiv = false;
};

namespace {
// relative FP64 residual above which block-local pivoting is abandoned
constexpr double kRefineFallback = 1e-10;
}

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}
}  // namespace

namespace {

int fail(necgpu_engine* e, int code, const std::string& msg) {
  e->err = msg;
  return code;
}

#define CUDA_TRY(call)                                                                         \
  do {                                                                                         \
    cudaError_t _st = (call);                                                                  \
    if (_st != cudaSuccess)                                                                    \
      return fail(e, NECGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_st));   \
  } while (0)

#define LAUNCHED()                                                                             \
  do {                                                                                         \
    e->launches++;                                                                             \
    cudaError_t _st = cudaGetLastError();                                                      \
    if (_st != cudaSuccess)                                                                    \
      return fail(e, NECGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(_st)); \
  } while (0)

#define TRY(x)           \
  do {                   \
    int _r = (x);        \
    if (_r) return _r;   \
  } while (0)

// Per-launch timing: an event pair on the launching stream around each
// kernel of a class, resolved after the next stream synchronisation.
int kbegin(necgpu_engine* e, cudaStream_t st = nullptr) {
  if (e->timing_level < 2) return -1;
  if (e->timing_level >= 3 && !e->trace_based) {
    // the trace's time origin: recorded before the first traced launch
    if (!e->trace_base && cudaEventCreate(&e->trace_base) != cudaSuccess) return -1;
    cudaEventRecord(e->trace_base, e->stream);
    e->trace_based = true;
  }
  while ((int)e->kev.size() < e->kev_used + 2) {
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return -1;
    e->kev.push_back(ev);
  }
  const int i = e->kev_used;
  e->kev_used += 2;
  cudaEventRecord(e->kev[i], st ? st : e->stream);
  return i;
}
void kend(necgpu_engine* e, int i, int cls, double flops, cudaStream_t st = nullptr, const char* name = nullptr) {
  if (i < 0) return;
  cudaStream_t s = st ? st : e->stream;
  cudaEventRecord(e->kev[i + 1], s);
  const int sid = s == e->stream ? 0 : s == e->stream2 ? 2 : s == e->stream3 ? 3 : s == e->stream4 ? 4 : 1;
  e->kpend.push_back({cls, i, flops, sid, name});
}
void kflush(necgpu_engine* e) {  // call after the stream has synchronised
  for (auto& p : e->kpend) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e->kev[p.ev], e->kev[p.ev + 1]) == cudaSuccess) {
      e->stats.k_ms[p.cls] += ms;
      e->stats.k_launches[p.cls] += 1;
      e->stats.k_flops[p.cls] += p.flops;
      float t0 = 0.f;
      if (e->timing_level >= 3 && e->trace_based &&
          cudaEventElapsedTime(&t0, e->trace_base, e->kev[p.ev]) == cudaSuccess && e->trace.size() < (1u << 20)) {
        necgpu_trace_rec r;
        r.cls = p.cls;
        r.stream = p.stream;
        r.start_ms = t0;
        r.end_ms = t0 + ms;
        r.work = p.flops;
        std::snprintf(r.name, sizeof r.name, "%s", p.name ? p.name : "");
        e->trace.push_back(r);
      }
    }
  }
  e->kpend.clear();
  e->kev_used = 0;
}

// launch a kernel of class cls (algorithmic work 'flops') and check it
#define KLAUNCH(cls, flops, ...)                         \
  do {                                                   \
    const int _kt = kbegin(e);                           \
    __VA_ARGS__;                                         \
    kend(e, _kt, (cls), (flops), nullptr, #__VA_ARGS__); \
    LAUNCHED();                                          \
  } while (0)

// launch with a scheduling priority (0: the stream's own); a CUDA graph
// captured from the stream keeps it on the kernel node
template <typename... KArgs, typename... Args>
cudaError_t launch_prio(int prio, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                        Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributePriority;
  attr[0].val.priority = prio;
  cfg.attrs = attr;
  cfg.numAttrs = prio ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

// Device buffers are stream-ordered allocations from the device's default
// memory pool, whose release threshold necgpu_create raises: memory freed by
// one engine (or one structure size) stays in the pool and serves the next
// allocation instead of being handed back to the driver and mapped again.
template <typename T>
void dfree(necgpu_engine* e, T*& p) {
  if (p) cudaFreeAsync((void*)p, e->stream);
  p = nullptr;
}

template <typename T>
int dalloc(necgpu_engine* e, T*& p, size_t count) {
  dfree(e, p);
  if (count == 0) count = 1;
  cudaError_t st = cudaMallocAsync((void**)&p, count * sizeof(T), e->stream);
  if (st != cudaSuccess) {
    p = nullptr;
    return fail(e, NECGPU_ERR_CUDA,
                std::string("cudaMallocAsync(") + std::to_string(count * sizeof(T)) + "): " + cudaGetErrorString(st));
  }
  return 0;
}

template <typename T>
int upload(necgpu_engine* e, T*& p, const T* h, size_t count) {
  TRY(dalloc(e, p, count));
  if (count) CUDA_TRY(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, e->stream));
  e->stats.h2d_bytes += count * sizeof(T);
  return 0;
}

void free_all(necgpu_engine* e) {
  if (e->lu_exec) {
    cudaGraphExecDestroy(e->lu_exec);
    e->lu_exec = nullptr;
  }
  e->lu_seen = LuGraphKey{};
  e->lu_key = LuGraphKey{};
  dfree(e, e->d_seg);
  dfree(e, e->d_ind);
  dfree(e, e->d_tile_ptr);
  dfree(e, e->d_tsrc);
  dfree(e, e->d_tsrc_eptr);
  dfree(e, e->d_ecol);
  dfree(e, e->d_ecoef);
  dfree(e, e->d_cptr);
  dfree(e, e->d_cbasis);
  dfree(e, e->d_ccoef);
  dfree(e, e->Z64);
  dfree(e, e->d_dinv);
  dfree(e, e->d_top_cnt);
  dfree(e, e->d_Bpan);
  e->bpan_bytes = 0;
  dfree(e, e->d_zload);
  dfree(e, e->d_somm);
  dfree(e, e->d_near_g);
  dfree(e, e->d_near_entry);
  dfree(e, e->d_near_rec);
  dfree(e, e->d_near_cols);
  e->somm_ready = false;
  e->near_g_cap = 0;
  e->near_cap = 0;
  dfree(e, e->d_Ap2);
  dfree(e, e->d_Bp2);
  dfree(e, e->d_Bp3);
  e->bp3_bytes = 0;
  e->tc_rows2 = 0;
  e->tc_kbytes2 = 0;
  dfree(e, e->d_tinv);
  dfree(e, e->d_sweep_ctr);
  dfree(e, e->ZT32);
  dfree(e, e->ZT64);
  dfree(e, e->d_tinvT);
  dfree(e, e->d_wnext);
  dfree(e, e->d_wnextT);
  dfree(e, e->d_adj_phi);
  dfree(e, e->d_adj_w);
  dfree(e, e->d_adj_r);
  e->adj_cap = 0;
  e->adj_ready = false;
  dfree(e, e->d_pseg);
  dfree(e, e->d_pecoef);
  dfree(e, e->d_pccoef);
  dfree(e, e->d_pout);
  dfree(e, e->d_pw);
  dfree(e, e->d_pfar);
  dfree(e, e->d_pargs);
  dfree(e, e->d_pcargs);
  dfree(e, e->d_pwts);
  e->p_cap = 0;
  e->pw_cap = 0;
  dfree(e, e->Z32);
  dfree(e, e->d_piv);
  dfree(e, e->d_src);
  dfree(e, e->d_perm);
  dfree(e, e->d_cand_val);
  dfree(e, e->d_cand_valf);
  dfree(e, e->d_cand_row);
  dfree(e, e->d_cand_rows);
  dfree(e, e->d_rowc);
  dfree(e, e->d_counter);
  dfree(e, e->d_b);
  dfree(e, e->d_x);
  dfree(e, e->d_r);
  dfree(e, e->d_cur);
  dfree(e, e->d_w1);
  dfree(e, e->d_w2);
  dfree(e, e->d_abc);
  dfree(e, e->d_rn2);
  dfree(e, e->d_theta);
  dfree(e, e->d_phi);
  dfree(e, e->d_eth);
  dfree(e, e->d_eph);
  dfree(e, e->d_flags);
  dfree(e, e->d_Ap);
  dfree(e, e->d_Bp);
  e->tc_rows = 0;
  e->tc_kbytes = 0;
  e->pat_cap = 0;
  e->res_ndir = 0;
  e->res_rhs = false;
  e->n = 0;
  e->factored = -1;
  e->filled = false;
}

void kflush(necgpu_engine* e);

int sync_status(necgpu_engine* e, int* out) {
  int h[4];
  CUDA_TRY(cudaMemcpyAsync(h, e->d_status, sizeof(h), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->stats.d2h_bytes += sizeof(h);
  kflush(e);
  *out = h[0];
  return 0;
}

void tick(necgpu_engine* e) {
  if (e->timing) cudaEventRecord(e->ev0, e->stream);
}
double tock(necgpu_engine* e) {
  if (!e->timing) return 0.0;
  cudaEventRecord(e->ev1, e->stream);
  cudaEventSynchronize(e->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e->ev0, e->ev1);
  return ms;
}

// ---------------- fill ----------------
template <int G, bool X>
int launch_fill_t(necgpu_engine* e, const FillArgs& a) {
  dim3 grid((unsigned)((e->n + kFillTI - 1) / kFillTI), (unsigned)e->ntiles);
  // work units of the fill: one per (observation, source) pair
  KLAUNCH(NECGPU_K_FILL, (double)e->n * (double)e->n,
          fill_kernel<G, X><<<grid, kFillTI, 0, e->stream>>>(a));
  return 0;
}

// Sommerfeld ground: evaluations that read the tables through the
// interpolation cache, in the reference's order over `nunits` units (source
// columns of the fill, or field points).  Every unit is first evaluated from
// a fresh cache, one thread per unit.  A unit's result depends on the cache
// it starts from only when its first table point falls below the cached
// patch's grid and the cached cell passes the reuse test; a host scan over
// the units in order finds those whose true starting cache (the one the
// previous unit leaves, the first unit starting from the cache the engine
// holds) differs from the one used, and only they are evaluated again from
// it.  The scan repeats until every unit is consistent; after a bounded
// number of rounds the rest is walked by one thread in order.  The cache
// left at the end is kept, with its coefficients, for the next evaluation.
// launch(entry, units, count, chain) runs the kernel; d_rec holds one
// NearRecord per unit.
template <typename Launch>
int resolve_cache_order(necgpu_engine* e, int64_t nunits, NearRecord* d_rec, Launch launch) {
  std::vector<InterpKey> entry((size_t)nunits, InterpKey{kInterpFresh, 0, 0, 0});
  std::vector<int> units((size_t)nunits);
  std::iota(units.begin(), units.end(), 0);
  std::vector<NearRecord> rec((size_t)nunits);
  if (!e->d_interp_carry) TRY(dalloc(e, e->d_interp_carry, 1));
  TRY(launch(entry, units, (int)nunits, 0));
  auto equal = [](InterpKey p, InterpKey q) {
    if (p.igrs == kInterpFresh || q.igrs == kInterpFresh) return p.igrs == q.igrs;
    return p.igrs == q.igrs && p.ix == q.ix && p.iy == q.iy && p.carry == q.carry;
  };
  const int kMaxRounds = 8;
  for (int round = 0;; round++) {
    CUDA_TRY(cudaMemcpyAsync(rec.data(), d_rec, (size_t)nunits * sizeof(NearRecord), cudaMemcpyDeviceToHost,
                             e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    InterpKey t = e->interp_key;
    int ndirty = 0, first_dirty = -1;
    for (int64_t j = 0; j < nunits; j++) {
      const NearRecord& r = rec[j];
      if (!r.has_near) continue;
      const InterpKey need = interp_reuses(t, r.x1, r.y1) ? t : InterpKey{kInterpFresh, 0, 0, 0};
      if (!equal(need, r.used)) {
        if (first_dirty < 0) first_dirty = (int)j;
        entry[j] = need;
        units[ndirty++] = (int)j;
      }
      t = r.exit;
    }
    e->stats.near_passes = round + 1;
    if (ndirty == 0) {
      if (t.igrs != kInterpFresh && !t.carry)
        KLAUNCH(NECGPU_K_FILL, 0.0, interp_store_kernel<<<1, 1, 0, e->stream>>>(t, e->d_somm, e->d_interp_carry));
      if (t.igrs != kInterpFresh) t.carry = 1;
      e->interp_key = t;
      return 0;
    }
    if (round > kMaxRounds) return fail(e, NECGPU_ERR_CUDA, "near-ground evaluation order did not settle");
    if (round + 1 < kMaxRounds) {
      TRY(launch(entry, units, ndirty, 0));
      continue;
    }
    // walk every unit from the first inconsistent one in order
    int m = 0;
    for (int64_t j = first_dirty; j < nunits; j++) units[m++] = (int)j;
    TRY(launch(entry, units, m, 1));
  }
}

// Near-ground pairs of the fill (pairs within the table limit of their
// image), one unit per source column in the reference's order (cmset).
template <bool X>
int run_near_ground(necgpu_engine* e, const FillArgs& a) {
  const int64_t n = e->n;
  if ((size_t)n * n * 3 > ((size_t)1 << 31))
    return fail(e, NECGPU_ERR_UNSUPPORTED, "fill: near-ground structures are limited to 26,000 segments");
  if (e->near_g_cap < n * n * 3) {
    dfree(e, e->d_near_g);
    TRY(dalloc(e, e->d_near_g, (size_t)n * n * 3));
    e->near_g_cap = n * n * 3;
  }
  if (e->near_cap < n) {
    TRY(dalloc(e, e->d_near_rec, (size_t)n));
    e->near_cap = n;
  }
  auto launch = [&](const std::vector<InterpKey>& entry, const std::vector<int>& cols, int ncols,
                    int chain) -> int {
    TRY(upload(e, e->d_near_entry, entry.data(), (size_t)n));
    TRY(upload(e, e->d_near_cols, cols.data(), (size_t)ncols));
    const unsigned blocks = chain ? 1u : (unsigned)((ncols + 63) / 64);
    KLAUNCH(NECGPU_K_FILL, 0.0,
            near_ground_kernel<X><<<blocks, chain ? 1 : 64, 0, e->stream>>>(
                a, e->d_somm, e->d_near_cols, ncols, e->d_near_entry, e->d_interp_carry, e->d_near_rec,
                e->d_near_g, chain));
    return 0;
  };
  return resolve_cache_order(e, n, e->d_near_rec, launch);
}

int run_fill(necgpu_engine* e, bool want64, bool want32) {
  if (e->n <= 0) return fail(e, NECGPU_ERR_ARG, "fill: no structure set");
  const int64_t n = e->n;
  if (want64 && !e->Z64) TRY(dalloc(e, e->Z64, (size_t)n * e->ld));
  if (want32 && !e->Z32) TRY(dalloc(e, e->Z32, (size_t)n * e->ld));
  FillArgs a{};
  a.n = n;
  a.ld = e->ld;
  a.x = e->d_seg;
  a.y = e->d_seg + n;
  a.z = e->d_seg + 2 * n;
  a.s = e->d_seg + 3 * n;
  a.b = e->d_seg + 4 * n;
  a.cab = e->d_seg + 5 * n;
  a.sab = e->d_seg + 6 * n;
  a.salp = e->d_seg + 7 * n;
  a.ind1 = e->d_ind;
  a.ind2 = e->d_ind + n;
  a.tile_src_ptr = e->d_tile_ptr;
  a.tsrc = e->d_tsrc;
  a.tsrc_eptr = e->d_tsrc_eptr;
  a.ecol = e->d_ecol;
  a.ea = e->d_ecoef;
  a.eb = e->d_ecoef + e->ne;
  a.ec = e->d_ecoef + 2 * e->ne;
  a.P = e->P;
  a.P.near_g = nullptr;
  a.Z64 = want64 ? e->Z64 : nullptr;
  a.Z32 = want32 ? e->Z32 : nullptr;
  a.status = e->d_status;
  const bool x = e->use_exk != 0;
  if (e->ground == kGroundSommerfeld && e->somm_ready) {
    TRY(x ? run_near_ground<true>(e, a) : run_near_ground<false>(e, a));
    a.P.near_g = e->d_near_g;
    a.P.near_n = n;
  }
  int rc;
  switch (e->ground) {
    case kGroundNone: rc = x ? launch_fill_t<kGroundNone, true>(e, a) : launch_fill_t<kGroundNone, false>(e, a); break;
    case kGroundPerfect:
      rc = x ? launch_fill_t<kGroundPerfect, true>(e, a) : launch_fill_t<kGroundPerfect, false>(e, a);
      break;
    case kGroundReflection:
      rc = x ? launch_fill_t<kGroundReflection, true>(e, a) : launch_fill_t<kGroundReflection, false>(e, a);
      break;
    default: rc = x ? launch_fill_t<kGroundSommerfeld, true>(e, a) : launch_fill_t<kGroundSommerfeld, false>(e, a);
  }
  if (rc) return rc;
  if (e->d_zload && want64)
    KLAUNCH(NECGPU_K_FILL, 0.0,
            load_kernel<<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(n, e->d_cptr, e->d_cbasis, e->d_ccoef,
                                                                            e->d_ccoef + 2 * e->nc, e->d_zload,
                                                                            e->Z64, e->ld));
  return 0;
}

template <int G, bool X>
int launch_near_e(necgpu_engine* e, const NearFieldArgs& a) {
  KLAUNCH(NECGPU_K_PATTERN, (double)a.npts * (double)e->n,
          near_e_kernel<G, X><<<(unsigned)((a.npts + kNearWarps - 1) / kNearWarps), 32 * kNearWarps, 0, e->stream>>>(a));
  return 0;
}

// ---------------- tensor-core trailing update ----------------
template <class F>
typename F::T* op(unsigned char* p) {
  return reinterpret_cast<typename F::T*>(p);
}

// Packed-operand buffers (set 0 or 1) sized for `rows` rows of up to `kdim`
// operand elements of format F (grown, never shrunk; sized in bytes, so
// either format fits once the larger was needed); the tensor maps are
// encoded per update for the update's own K'.
template <class F>
int ensure_tc(necgpu_engine* e, int kdim, int64_t rows, int set = 0) {
  if (!(e->tc_attr & F::kFormat)) {
    CUDA_TRY(cudaFuncSetAttribute(tc::gemm_tc_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    e->tc_attr |= F::kFormat;
  }
  unsigned char*& Ap = set ? e->d_Ap2 : e->d_Ap;
  unsigned char*& Bp = set ? e->d_Bp2 : e->d_Bp;
  int64_t& trows = set ? e->tc_rows2 : e->tc_rows;
  int64_t& tkb = set ? e->tc_kbytes2 : e->tc_kbytes;
  const int64_t kbytes = (int64_t)kdim * (int64_t)sizeof(typename F::T);
  if (Ap && trows >= rows && tkb >= kbytes) return 0;
  if (!encode_tiled()) return fail(e, NECGPU_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const int64_t r = std::max(rows, trows);
  const int64_t k = std::max(kbytes, tkb);
  TRY(dalloc(e, Ap, (size_t)(r * k)));
  TRY(dalloc(e, Bp, (size_t)(2 * r * k)));
  trows = r;
  tkb = k;
  return 0;
}

// K-major operand map of format F: nrows rows of kdim elements, boxes of 128
// bytes x box_rows
template <class F>
int encode_operand(necgpu_engine* e, CUtensorMap* map, void* base, int kdim, int64_t nrows, uint32_t box_rows) {
  cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)nrows};
  cuuint64_t strides[1] = {(cuuint64_t)kdim * sizeof(typename F::T)};
  cuuint32_t box[2] = {(cuuint32_t)tc::bk<F>(), box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt =
      F::kFormat == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  CUresult r = encode_tiled()(map, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : fail(e, NECGPU_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

// Pack A (m x kb) and B (kb x n), complex64 row-major with leading
// dimension ld, into operand set `set` (on the engine's stream).
template <class F>
int tc_pack(necgpu_engine* e, int set, const float2* A, const float2* B, int64_t ld, int64_t m, int64_t n, int kb,
            bool pack_b = true) {
  const int kbp = (kb + tc::KP - 1) / tc::KP * tc::KP;
  TRY(ensure_tc<F>(e, F::kKMul * kbp, std::max(m, n), set));
  typename F::T* Ap = op<F>(set ? e->d_Ap2 : e->d_Ap);
  typename F::T* Bp = op<F>(set ? e->d_Bp2 : e->d_Bp);
  const int64_t cnt = m * kbp;
  KLAUNCH(NECGPU_K_OTHER, 0.0,
          tc::pack_a_kernel<F><<<(unsigned)((cnt + 255) / 256), 256, 0, e->stream>>>(A, ld, (int)m, kb, kbp, Ap));
  if (!pack_b) return 0;
  dim3 g((unsigned)((n + 31) / 32), (unsigned)(kbp / 64));
  KLAUNCH(NECGPU_K_OTHER, 0.0, tc::pack_b_kernel<F><<<g, 256, 0, e->stream>>>(B, ld, kb, kbp, (int)n, Bp));
  return 0;
}

// C (m x ncols) -= A' B'[columns j0, j0 + ncols) from operand set `set`, on
// stream st with at most grid_max persistent CTAs.
template <class F>
int tc_run(necgpu_engine* e, int set, int64_t m, int64_t j0, int64_t ncols, int kb, float2* C, int64_t ld,
           cudaStream_t st, int grid_max, int64_t a_row0 = 0, typename F::T* Bp_alt = nullptr) {
  const int kbp = (kb + tc::KP - 1) / tc::KP * tc::KP;
  const int kdim = F::kKMul * kbp;
  typename F::T* Ap = op<F>(set ? e->d_Ap2 : e->d_Ap) + a_row0 * kdim;
  typename F::T* Bp = Bp_alt ? Bp_alt : op<F>(set ? e->d_Bp2 : e->d_Bp);
  CUtensorMap tmA, tmB, tmC;
  TRY(encode_operand<F>(e, &tmA, Ap, kdim, m, tc::BM));
  TRY(encode_operand<F>(e, &tmB, Bp + 2 * j0 * kdim, kdim, 2 * ncols, tc::BN));
  // C as m rows x 2 ncols FP32 (re, im interleaved), 32 x 32 boxes for the
  // reduce-add epilogue; TMA clips the boxes at the edges of C
  {
    cuuint64_t dims[2] = {(cuuint64_t)(2 * ncols), (cuuint64_t)m};
    cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float2)};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_tiled()(&tmC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)C, dims, strides, box, estr,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
      return fail(e, NECGPU_ERR_CUDA, "cuTensorMapEncodeTiled (C) failed: " + std::to_string((int)r));
  }
  const int m_tiles = (int)((m + tc::BM - 1) / tc::BM);
  const int n_tiles = (int)((2 * ncols + tc::BN - 1) / tc::BN);
  const int grid = std::max(1, std::min(m_tiles * n_tiles, grid_max));
  const int kt = kbegin(e, st);
  const int group = std::max(1, std::min(e->gemm_group, m_tiles));
  tc::gemm_tc_kernel<F><<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(tmA, tmB, tmC, (int)m, (int)ncols, kdim,
                                                                  group, e->d_status);
  kend(e, kt, NECGPU_K_GEMM, 8.0 * (double)m * ncols * kb, st, "tc::gemm_tc_kernel");
  LAUNCHED();
  return 0;
}

// C (m x n) -= A (m x kb) B (kb x n), complex64 row-major with leading
// dimension ld, on the tensor cores (operand set 0, whole device).
template <class F>
int tc_gemm_sub(necgpu_engine* e, const float2* A, const float2* B, float2* C, int64_t ld, int64_t m, int64_t n,
                int kb, int grid_max = 0) {
  TRY(tc_pack<F>(e, 0, A, B, ld, m, n, kb));
  return tc_run<F>(e, 0, m, 0, n, kb, C, ld, e->stream, grid_max > 0 ? grid_max : e->nsm);
}

// trailing update of the FP32 LU for the panel at k0 of width kb
template <class F>
int tc_update(necgpu_engine* e, float2* M, int64_t k0, int kb) {
  const int64_t ld = e->ld, r0 = k0 + kb, rest = e->n - r0;
  return tc_gemm_sub<F>(e, M + r0 * ld + k0, M + k0 * ld + r0, M + r0 * ld + r0, ld, rest, rest, kb);
}

__global__ void fill_random_kernel(float2* p, int64_t count, uint32_t seed) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t h = (uint32_t)i * 2654435761u ^ seed;
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  h ^= h >> 16;
  uint32_t g = h * 1664525u + 1013904223u;
  p[i] = make_float2((h & 0xffffff) / 16777216.0f - 0.5f, (g & 0xffffff) / 16777216.0f - 0.5f);
}

__global__ void max_diff_kernel(const float2* a, const float2* b, int64_t ld, int64_t m, int64_t n, float* out) {
  float mx = 0.f, ref = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m * n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = i / n, c = i - r * n;
    float2 x = a[r * ld + c], y = b[r * ld + c];
    mx = fmaxf(mx, fmaxf(fabsf(x.x - y.x), fabsf(x.y - y.y)));
    ref = fmaxf(ref, fmaxf(fabsf(y.x), fabsf(y.y)));
  }
  atomicMax((int*)out, __float_as_int(mx));
  atomicMax((int*)out + 1, __float_as_int(ref));
}

// ---------------- LU ----------------
template <typename R, class F = tc::SplitBf16>
int run_lu(necgpu_engine* e, typename cvec<R>::T* M) {
  using T = typename cvec<R>::T;
  const int64_t n = e->n, ld = e->ld;
  if (!e->d_piv) TRY(dalloc(e, e->d_piv, (size_t)n));
  const int Pmax = e->nsm;
  if (!e->d_cand_val) TRY(dalloc(e, e->d_cand_val, 2 * (size_t)Pmax));
  if (!e->d_cand_valf) TRY(dalloc(e, e->d_cand_valf, 2 * (size_t)Pmax));
  if (!e->d_cand_row) TRY(dalloc(e, e->d_cand_row, 2 * (size_t)Pmax));
  if (!e->d_cand_rows) TRY(dalloc(e, e->d_cand_rows, 2 * (size_t)Pmax * kNB));
  if (!e->d_rowc) TRY(dalloc(e, e->d_rowc, 2 * (size_t)kNB));
  if (!e->d_counter) TRY(dalloc(e, e->d_counter, 1));

  constexpr size_t kSmemLimit = 200 * 1024;
  const size_t row_bytes = kNB * sizeof(T);
  const int rpc_max = (int)((kSmemLimit - 2 * row_bytes) / row_bytes);
  CUDA_TRY(cudaFuncSetAttribute(panel_kernel<R, kNB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSmemLimit));
  const size_t trsm_smem = (size_t)(kNB * kNB + kNB * 32) * sizeof(T);
  CUDA_TRY(cudaFuncSetAttribute(trsm_kernel<T, kNB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm_smem));

  PanelArgs<R> pa{};
  pa.M = M;
  pa.ld = ld;
  pa.n = n;
  pa.piv = e->d_piv;
  pa.cand_val = std::is_same<R, double>::value ? (R*)e->d_cand_val : (R*)e->d_cand_valf;
  pa.cand_row = e->d_cand_row;
  pa.cand_rows = (T*)e->d_cand_rows;
  pa.rowc = (T*)e->d_rowc;
  pa.counter = e->d_counter;
  pa.status = e->d_status;

  for (int64_t k0 = 0; k0 < n; k0 += kNB) {
    const int kb = (int)std::min<int64_t>(kNB, n - k0);
    const int64_t m = n - k0;
    int P = (int)std::min<int64_t>(Pmax, (m + 15) / 16);
    P = std::max(P, 1);
    int rpc = (int)((m + P - 1) / P);
    if (rpc > rpc_max) return fail(e, NECGPU_ERR_UNSUPPORTED, "LU: panel does not fit in shared memory");
    P = (int)((m + rpc - 1) / rpc);
    pa.k0 = k0;
    pa.kb = kb;
    pa.rpc = rpc;
    const size_t smem = (size_t)rpc * row_bytes + 2 * row_bytes;
    CUDA_TRY(cudaMemsetAsync(e->d_counter, 0, sizeof(unsigned), e->stream));
    void* args[] = {&pa};
    {
      // panel: m x kb unblocked LU, ~8 m kb^2 / 2 real flops
      const int kt = kbegin(e);
      CUDA_TRY(cudaLaunchCooperativeKernel((const void*)panel_kernel<R, kNB>, dim3(P), dim3(kPanelThreads),
                                           args, smem, e->stream));
      kend(e, kt, NECGPU_K_PANEL, 4.0 * (double)m * kb * kb, nullptr, "trsm_panel_kernel");
      LAUNCHED();
    }
    if (n > kb)
      KLAUNCH(NECGPU_K_LASWP, 0.0,
              laswp_kernel<T><<<(unsigned)((n + 255) / 256), 256, 0, e->stream>>>(M, ld, n, k0, kb, e->d_piv));
    const int64_t rest = n - k0 - kb;
    if (rest > 0) {
      KLAUNCH(NECGPU_K_TRSM, 4.0 * (double)kb * kb * rest,
              trsm_kernel<T, kNB><<<(unsigned)((rest + 31) / 32), 256, trsm_smem, e->stream>>>(M, ld, n, k0, kb));
      bool done = false;
      if constexpr (std::is_same<R, float>::value) {
        if (e->use_tc) {
          TRY(tc_update<F>(e, M, k0, kb));
          done = true;
        }
      }
      if constexpr (std::is_same<R, double>::value) {
        if (!done && e->use_dmma) {
          // FP64 tensor cores (mma.sync m8n8k4 f64)
          dim3 g((unsigned)((rest + kDmmaBN - 1) / kDmmaBN), (unsigned)((rest + kDmmaBM - 1) / kDmmaBM));
          KLAUNCH(NECGPU_K_GEMM, 8.0 * (double)rest * rest * kb,
                  gemm_dmma_kernel<<<g, kDmmaThreads, sizeof(DmmaSmem), e->stream>>>(
                      M + (k0 + kb) * ld + k0, ld, M + k0 * ld + k0 + kb, ld, M + (k0 + kb) * ld + k0 + kb, ld, rest,
                      rest, kb));
          done = true;
        }
      }
      if (!done) {
        dim3 g((unsigned)((rest + 63) / 64), (unsigned)((rest + 63) / 64));
        // complex multiply-add = 8 real flops
        KLAUNCH(NECGPU_K_GEMM, 8.0 * (double)rest * rest * kb,
                gemm_sub_kernel<R><<<g, 256, 0, e->stream>>>(M + (k0 + kb) * ld + k0, ld, M + k0 * ld + k0 + kb,
                                                             ld, M + (k0 + kb) * ld + k0 + kb, ld, rest, rest, kb));
      }
    }
  }
  // permutation of the right-hand side from the interchange sequence
  std::vector<int> piv(n), perm(n);
  CUDA_TRY(cudaMemcpyAsync(piv.data(), e->d_piv, n * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += n * sizeof(int);
  int st = 0;
  TRY(sync_status(e, &st));
  for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
  for (int64_t k = 0; k < n; k++) {
    int p = piv[k];
    if (p < 0 || p >= n) return fail(e, NECGPU_ERR_NONFINITE, "LU: invalid pivot index");
    std::swap(perm[k], perm[p]);
  }
  TRY(upload(e, e->d_perm, perm.data(), perm.size()));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (st & kLuStatBarrierTimeout) return fail(e, NECGPU_ERR_CUDA, "LU: panel barrier timed out");
  if (st & tc::kStatTimeout) return fail(e, NECGPU_ERR_CUDA, "LU: tensor-core update pipeline timed out");
  if (st & kLuStatNonFinite) return fail(e, NECGPU_ERR_NONFINITE, "LU: NaN/Inf in the matrix");
  if (st & kLuStatSingular) return fail(e, NECGPU_ERR_SINGULAR, "LU: singular matrix (zero pivot)");
  return 0;
}

// FP32 LU with block-local pivoting (mixed path): per 64-column panel, one
// CTA factors the diagonal block, the exchanges are a per-column gather
// inside the block, L21 and U12 are row/column-parallel triangular solves,
// and the trailing update runs on the tensor cores.
template <class F>
int run_lu_blockpiv(necgpu_engine* e, float2* M) {
  using T = float2;
  using Op = typename F::T;  // packed operand element
  const int64_t n = e->n, ld = e->ld;
  const int64_t nblk = (n + kBlk - 1) / kBlk;
  if (!e->d_piv) TRY(dalloc(e, e->d_piv, (size_t)n));
  if (!e->d_src) TRY(dalloc(e, e->d_src, (size_t)n));
  if (!e->d_dinv) TRY(dalloc(e, e->d_dinv, (size_t)nblk * kBlk));
  CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm_panel_smem<T>()));
  CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm_panel_smem<T>()));
  CUDA_TRY(cudaFuncSetAttribute(trsm_panel_kernel<T, false, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm_panel_smem<T>()));
  CUDA_TRY(cudaFuncSetAttribute(trsm8_panel_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm8_smem<T>()));
  CUDA_TRY(cudaFuncSetAttribute(trsm8_panel_kernel<T, true, 1, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)trsm8_smem<T>()));
  CUDA_TRY(cudaFuncSetAttribute(panel_top_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)panel_top_smem()));
  CUDA_TRY(cudaFuncSetAttribute(l21_rows_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)l21_rows_smem()));
  // panel solve: vectors [sbeg, nend) against the 64 x 64 block at k0
  // (LEFT: columns of U12, else rows of L21); kind and flop count for timing
  auto trsm = [&](bool left, int64_t k0, int64_t sbeg, int64_t nend, const T* dinv, int kind,
                  Op* Ap = nullptr, int64_t abase = 0) -> int {
    const int64_t cnt = nend - sbeg;
    if (cnt <= 0) return 0;
    const double fl = 4.0 * (double)kBlk * kBlk * cnt;
    // eight warps per block of 32 vectors pay off for the U12 columns
    // (coalesced along the row); the L21 rows stay one per thread, which
    // measured faster than the eight-warp form with 32 or 128 rows per CTA
    if (e->trsm8 && left) {
      const unsigned g = (unsigned)((cnt + kTrsm8Vec - 1) / kTrsm8Vec);
      KLAUNCH(kind, fl, trsm8_panel_kernel<T, true><<<g, 256, (unsigned)trsm8_smem<T>(), e->stream>>>(
                            M, ld, nend, k0, sbeg, dinv));
      return 0;
    }
    if (!left && e->l21_rows) {
      const unsigned g = (unsigned)std::min<int64_t>((cnt + kL21Rows - 1) / kL21Rows, 4 * (int64_t)e->nsm);
      KLAUNCH(kind, fl, l21_rows_kernel<F><<<g, 256, (unsigned)l21_rows_smem(), e->stream>>>(M, ld, nend, k0, sbeg, dinv,
                                                                                            Ap, abase));
      return 0;
    }
    const unsigned g = (unsigned)((cnt + kTrsmW - 1) / kTrsmW);
    const unsigned sm = (unsigned)trsm_panel_smem<T>();
    if (left)
      KLAUNCH(kind, fl, trsm_panel_kernel<T, true><<<g, kTrsmW, sm, e->stream>>>(M, ld, nend, k0, sbeg, dinv));
    else
      KLAUNCH(kind, fl,
              trsm_panel_kernel<T, false, F><<<g, kTrsmW, sm, e->stream>>>(M, ld, nend, k0, sbeg, dinv, Ap, abase));
    return 0;
  };
  // U12 of an inner panel (eight-warp form) on stream st
  auto trsm_left_on = [&](int64_t k0, int64_t sbeg, int64_t nend, const T* dinv, int kind, cudaStream_t st,
                          Op* Bp = nullptr, int64_t bbase = 0) -> int {
    const int64_t cnt = nend - sbeg;
    if (cnt <= 0) return 0;
    const unsigned g = (unsigned)((cnt + kTrsm8Vec - 1) / kTrsm8Vec);
    const int kt = kbegin(e, st);
    trsm8_panel_kernel<T, true, 1, F><<<g, 256, (unsigned)trsm8_smem<T>(), st>>>(M, ld, nend, k0, sbeg, dinv, Bp,
                                                                                bbase);
    kend(e, kt, kind, 4.0 * (double)kBlk * kBlk * cnt, st, "trsm8_panel_kernel");
    LAUNCHED();
    return 0;
  };
  // L21 rows [sbeg, nend) of the panel at k0 (one row per thread) on stream st
  auto trsm_on = [&](int64_t k0, int64_t sbeg, int64_t nend, const T* dinv, int kind, cudaStream_t st,
                     Op* Ap, int64_t abase) -> int {
    const int64_t cnt = nend - sbeg;
    if (cnt <= 0) return 0;
    const int kt = kbegin(e, st);
    if (e->l21_rows) {
      // a capped persistent grid: this solve runs beside the panel chain
      const unsigned g = (unsigned)std::min<int64_t>((cnt + kL21Rows - 1) / kL21Rows, e->side_ctas);
      l21_rows_kernel<F><<<g, 256, (unsigned)l21_rows_smem(), st>>>(M, ld, nend, k0, sbeg, dinv, Ap, abase);
      kend(e, kt, kind, 4.0 * (double)kBlk * kBlk * cnt, st, "l21_rows_kernel");
    } else {
      const unsigned g = (unsigned)((cnt + kTrsmW - 1) / kTrsmW);
      trsm_panel_kernel<T, false, F><<<g, kTrsmW, (unsigned)trsm_panel_smem<T>(), st>>>(M, ld, nend, k0, sbeg,
                                                                                        dinv, Ap, abase);
      kend(e, kt, kind, 4.0 * (double)kBlk * kBlk * cnt, st, "trsm_panel_kernel");
    }
    LAUNCHED();
    return 0;
  };
  if (e->trsm8 && !e->stream3) {
    CUDA_TRY(cudaStreamCreateWithFlags(&e->stream3, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_u12a, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_u12b, cudaEventDisableTiming));
  }
  // gemm_grid: CTAs the persistent tensor-core update may take (fewer while
  // a far update runs beside the panel work)
  int gemm_grid = e->nsm;
  auto gemm = [&](int64_t r0, int64_t c0, int64_t kc, int64_t m, int64_t nc, int kk) -> int {
    // M[r0.., c0..] (m x nc) -= M[r0.., kc..kc+kk) M[kc..kc+kk, c0..)
    if (m <= 0 || nc <= 0 || kk <= 0) return 0;
    if (e->use_tc)
      return tc_gemm_sub<F>(e, M + r0 * ld + kc, M + kc * ld + c0, M + r0 * ld + c0, ld, m, nc, kk, gemm_grid);
    dim3 gg((unsigned)((nc + 63) / 64), (unsigned)((m + 63) / 64));
    KLAUNCH(NECGPU_K_GEMM, 8.0 * (double)m * nc * kk,
            gemm_sub_kernel<float><<<gg, 256, 0, e->stream>>>(M + r0 * ld + kc, ld, M + kc * ld + c0, ld,
                                                              M + r0 * ld + c0, ld, m, nc, kk));
    return 0;
  };
  // interchanges of the panel at k0 on columns [c_lo, c_hi) outside
  // [k0, skip_hi) (default: the diagonal block), on stream st
  auto laswp = [&](int64_t k0, int kb, int64_t c_lo, int64_t c_hi, cudaStream_t st = nullptr,
                   int64_t skip_hi = -1) -> int {
    if (c_hi <= c_lo) return 0;
    cudaStream_t s = st ? st : e->stream;
    const int kt = kbegin(e, s);
    laswp_block_kernel<T><<<(unsigned)((c_hi - c_lo + 31) / 32), 256, 0, s>>>(M, ld, c_lo, c_hi, k0, kb, e->d_src,
                                                                             skip_hi < 0 ? k0 + kb : skip_hi);
    kend(e, kt, NECGPU_K_LASWP, 0.0, s, "laswp_block_kernel<T>");
    LAUNCHED();
    return 0;
  };
  // Outer blocks of e->outer columns (a multiple of 64) factored with 64-wide
  // inner panels whose updates stay inside the outer block's columns; the
  // outer block's U12 rows are brought up to date left-looking, and one
  // tensor-core update with K = outer covers the trailing matrix.
  //
  // Lookahead: that trailing update is split.  Its first `outer` columns
  // (the next outer block) are updated at once; the rest (the far update)
  // runs on stream2 with lookahead_sms SMs left free, while the next outer
  // block's panels are factored.  Those panels' row interchanges reach only
  // columns left of the far update; the far columns get them after the far
  // update has finished, before the next U12 rows are formed.
  const int64_t outer = e->outer;
  const bool la = e->lookahead && e->use_tc && e->nsm > 2 * e->lookahead_sms;
  if (la && !e->stream2) {
    CUDA_TRY(cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_far, cudaEventDisableTiming));
  }
  // the outer row block's U12 in one launch (u12_rows_kernel) when its
  // finished rows fit in shared memory and its 64-row blocks are whole
  const bool u12_fused = e->u12_fused && outer % kBlk == 0 && outer / kBlk <= kU12MaxBlocks;
  const bool fused_pack = e->fused_pack && e->use_tc;
  // each inner panel's L21 solve and update split at the next panel's rows:
  // the part that the next diagonal LU needs on the engine's stream, the
  // rest on stream4 beside it
  const bool split_inner = e->inner_split && fused_pack && e->trsm8;
  if (split_inner && !e->stream4) {
    CUDA_TRY(cudaStreamCreateWithFlags(&e->stream4, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_diag, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_bulk, cudaEventDisableTiming));
  }
  // the split panels' next-block rows in one launch (panel_top_kernel),
  // their interchanges on stream3
  const bool panel_top = split_inner && e->panel_top && e->stream3 && outer >= 2 * kBlk &&
                         (outer - kBlk) / kTopRows <= kTopRowGroups &&
                         kTopRowGroups + (outer - kBlk) / kTopCols <= kTopCnt;
  // B operand slots of panel_top_kernel, one per panel of an outer block
  const size_t bpan_slot = 2 * (size_t)(outer - kBlk) * F::kKMul * kBlk;  // elements
  if (panel_top && !e->ev_swap) CUDA_TRY(cudaEventCreateWithFlags(&e->ev_swap, cudaEventDisableTiming));
  if (panel_top && !e->d_top_cnt) {
    TRY(dalloc(e, e->d_top_cnt, (size_t)kTopCnt));
    CUDA_TRY(cudaMemsetAsync(e->d_top_cnt, 0, kTopCnt * sizeof(unsigned), e->stream));
  }
  if (panel_top) {
    const size_t need = (size_t)(outer / kBlk - 1) * bpan_slot * sizeof(Op);
    if (!e->d_Bpan || e->bpan_bytes < need) {
      TRY(dalloc(e, e->d_Bpan, need));
      e->bpan_bytes = need;
    }
  }
  if (u12_fused)
    CUDA_TRY(cudaFuncSetAttribute(u12_rows_kernel<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)u12_rows_smem((int)(outer / kBlk))));
  // the whole factorisation on the device, as launches on the engine's
  // stream (and stream2 / stream3, joined back into it)
  auto issue = [&]() -> int {
    bool far_pending = false;
    for (int64_t K0 = 0; K0 < n; K0 += outer) {
      const int64_t KE = std::min<int64_t>(n, K0 + outer);  // end of the outer block
      const int64_t swap_hi = far_pending ? KE : n;          // columns the far update is not touching
      gemm_grid = far_pending ? e->lookahead_sms : e->nsm;
      bool bulk_pending = false;  // stream4 holds the last panel's work below the next panel's rows
      bool swap_pending = false;  // stream3 holds interchanges of this block's panels
      for (int64_t k0 = K0; k0 < KE; k0 += kBlk) {
        const int kb = (int)std::min<int64_t>(kBlk, n - k0);
        T* dinv = e->d_dinv + k0;
        {
          const int kt = kbegin(e);
          CUDA_TRY(launch_prio(e->chain_prio, diag_lu_kernel<T>, dim3(1), dim3(kDiagThreads), 0, e->stream, M, ld, k0,
                               kb, e->d_piv, e->d_src, dinv, e->d_status));
          kend(e, kt, NECGPU_K_PANEL, 8.0 * (double)kb * kb * kb / 3.0, nullptr, "diag_lu_kernel<T>");
          LAUNCHED();
        }
        const int64_t r0 = k0 + kb, rest = n - r0;
        const int64_t pc = KE - r0;  // panel columns of this outer block right of the inner panel
        if (panel_top && kb == kBlk) {
          // Block rows and columns on this stream, one launch per panel: the
          // rest of the outer block's rows take their L21 rows, this panel's
          // U12 (the interchanges gathered as it loads) and their update in
          // panel_top_kernel.  The rows below the outer block take their L21
          // rows and update on stream4, needed only by the trailing update;
          // the panel's interchanges on the other columns go to stream3.
          // Each panel of the block has its own B operand slot, so this
          // stream never waits for stream4.
          CUDA_TRY(cudaEventRecord(e->ev_diag, e->stream));  // U11, its reciprocal diagonal and the row order
          if (n > kb) {
            CUDA_TRY(cudaStreamWaitEvent(e->stream3, e->ev_diag, 0));
            TRY(laswp(k0, kb, 0, swap_hi, e->stream3, KE));
            swap_pending = true;
          }
          if (rest <= 0) continue;
          const int64_t below = n - KE;
          if (below > 0) {
            CUDA_TRY(cudaStreamWaitEvent(e->stream4, e->ev_diag, 0));
            TRY(trsm_on(k0, KE, n, dinv, NECGPU_K_PANEL, e->stream4, pc > 0 ? op<F>(e->d_Ap) : nullptr, KE));
          }
          if (pc > 0) {
            Op* Bsel = op<F>(e->d_Bpan) + (size_t)((k0 - K0) / kBlk) * bpan_slot;
            const dim3 tg((unsigned)((pc + kTopCols - 1) / kTopCols), (unsigned)((pc + kTopRows - 1) / kTopRows));
            const int kt = kbegin(e);
            CUDA_TRY(launch_prio(e->chain_prio, panel_top_kernel<F>, tg, dim3(kTopThreads), panel_top_smem(), e->stream,
                                 M, ld, k0, KE, (const int*)e->d_src, (const float2*)dinv, Bsel, e->d_top_cnt));
            kend(e, kt, NECGPU_K_TRSM, (4.0 * kBlk * kBlk + 8.0 * kBlk * (double)pc) * 2.0 * (double)pc, nullptr,
                 "panel_top_kernel");
            LAUNCHED();
            if (below > 0) {
              CUDA_TRY(cudaEventRecord(e->ev_u12b, e->stream));
              CUDA_TRY(cudaStreamWaitEvent(e->stream4, e->ev_u12b, 0));
              TRY(tc_run<F>(e, 0, below, 0, pc, kb, M + KE * ld + r0, ld, e->stream4,
                         std::min(gemm_grid, e->side_ctas), 0, Bsel));
            }
          }
          if (below > 0) {
            CUDA_TRY(cudaEventRecord(e->ev_bulk, e->stream4));
            bulk_pending = true;
          }
          continue;
        }
        const bool split = split_inner && kb == kBlk && pc > 0 && rest > 2 * kBlk;
        if (split) CUDA_TRY(cudaEventRecord(e->ev_diag, e->stream));  // U11 and its reciprocal diagonal are ready
        if (n > kb) TRY(laswp(k0, kb, 0, swap_hi));
        if (rest <= 0) continue;
        if (split) {
          // Rows [r0, r0 + 64) (the next diagonal block's) take their L21
          // rows and update on this stream; the rows below take theirs on
          // stream4, beside the next diagonal LU.  The A operand's rows are
          // split the same way; the B operand alternates between two
          // buffers so that U12 of the next panel never overwrites the one
          // the bulk update is reading.
          const int p = (int)((k0 - K0) / kBlk);
          Op* Bsel = op<F>((p & 1) ? e->d_Bp3 : e->d_Bp);
          CUDA_TRY(cudaEventRecord(e->ev_u12a, e->stream));
          CUDA_TRY(cudaStreamWaitEvent(e->stream3, e->ev_u12a, 0));
          TRY(trsm_left_on(k0, r0, KE, dinv, NECGPU_K_TRSM, e->stream3, Bsel, r0));
          CUDA_TRY(cudaEventRecord(e->ev_u12b, e->stream3));
          // the bulk: L21 rows [r0 + 64, n) after the diagonal LU, then their update
          CUDA_TRY(cudaStreamWaitEvent(e->stream4, e->ev_diag, 0));
          TRY(trsm_on(k0, r0 + kBlk, n, dinv, NECGPU_K_PANEL, e->stream4, op<F>(e->d_Ap), r0));
          CUDA_TRY(cudaStreamWaitEvent(e->stream4, e->ev_u12b, 0));
          TRY(tc_run<F>(e, 0, rest - kBlk, 0, pc, kb, M + (r0 + kBlk) * ld + r0, ld, e->stream4, gemm_grid, kBlk,
                     Bsel));
          // the next diagonal block's rows: their L21 rows need the previous
          // bulk update (it reached them), then their update
          if (bulk_pending) CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_bulk, 0));
          TRY(trsm(false, k0, r0, r0 + kBlk, dinv, NECGPU_K_PANEL, op<F>(e->d_Ap), r0));
          CUDA_TRY(cudaEventRecord(e->ev_bulk, e->stream4));
          bulk_pending = true;
          CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_u12b, 0));
          TRY(tc_run<F>(e, 0, kBlk, 0, pc, kb, M + r0 * ld + r0, ld, e->stream, gemm_grid, 0, Bsel));
          continue;
        }
        if (bulk_pending) {  // rows below this panel were last updated on stream4
          CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_bulk, 0));
          bulk_pending = false;
        }
        // U12 (rows of the block, columns [r0, KE)) and L21 (rows [r0, n),
        // the block's columns) touch disjoint parts of M: U12 runs on stream3
        // beside L21, and the update after them waits for both
        const bool fork = pc > 0 && e->trsm8 && e->stream3;
        // the two panel solves write the update's packed BF16 operands
        // (operand set 0) as they store their results: no packing passes
        const bool emit = fork && fused_pack && kb == kBlk;
        if (fork) {
          CUDA_TRY(cudaEventRecord(e->ev_u12a, e->stream));
          CUDA_TRY(cudaStreamWaitEvent(e->stream3, e->ev_u12a, 0));
          TRY(trsm_left_on(k0, r0, KE, dinv, NECGPU_K_TRSM, e->stream3, emit ? op<F>(e->d_Bp) : nullptr, r0));
          CUDA_TRY(cudaEventRecord(e->ev_u12b, e->stream3));
        }
        TRY(trsm(false, k0, r0, n, dinv, NECGPU_K_PANEL, emit ? op<F>(e->d_Ap) : nullptr, r0));
        if (pc > 0) {
          if (fork)
            CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_u12b, 0));
          else
            TRY(trsm(true, k0, r0, KE, dinv, NECGPU_K_TRSM));
          if (emit)
            TRY(tc_run<F>(e, 0, rest, 0, pc, kb, M + r0 * ld + r0, ld, e->stream, gemm_grid));
          else
            TRY(gemm(r0, r0, k0, rest, pc, kb));
        }
      }
      // (with panel_top_kernel the rows below the outer block are needed
      // only by the trailing update, and U12 of the row block goes ahead)
      if (bulk_pending && !panel_top) CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_bulk, 0));
      if (swap_pending) {
        CUDA_TRY(cudaEventRecord(e->ev_swap, e->stream3));
        CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_swap, 0));
      }
      gemm_grid = e->nsm;
      // the far columns still owe this block's interchanges when the far
      // update of the previous block ran beside its panels
      const bool swap_far = far_pending;
      if (far_pending) {
        CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_far, 0));
        far_pending = false;
      }
      const int64_t rest = n - KE;
      const int nbo = (int)((KE - K0) / kBlk);
      // the fused U12 also writes the trailing update's packed B operand
      // (set 1, free: the far update that read it has finished) when the
      // lookahead path below is taken
      const bool u12_emit = u12_fused && fused_pack && la && rest > outer && KE - K0 == outer;
      if (rest > 0 && u12_fused) {
        // U12 of the outer row block, rows [K0, KE) x columns [KE, n), with
        // the far columns' interchanges, in one launch
        KLAUNCH(NECGPU_K_TRSM, 4.0 * (double)(KE - K0) * (double)(KE - K0) * (double)rest,
                u12_rows_kernel<F><<<(unsigned)((rest + kU12Cols - 1) / kU12Cols), 256, (unsigned)u12_rows_smem(nbo),
                                  e->stream>>>(
                    M, ld, K0, nbo, KE, n, e->d_src, swap_far ? 1 : 0, u12_emit ? op<F>(e->d_Bp2) : nullptr));
      } else {
        if (swap_far)
          for (int64_t k0 = K0; k0 < KE; k0 += kBlk) TRY(laswp(k0, (int)std::min<int64_t>(kBlk, n - k0), KE, n));
        if (rest <= 0) continue;
        // U12 of the outer row block: rows [K0, KE), columns [KE, n)
        for (int64_t k0 = K0; k0 < KE; k0 += kBlk) {
          TRY(gemm(k0, KE, K0, kBlk, rest, (int)(k0 - K0)));
          TRY(trsm(true, k0, KE, n, e->d_dinv + k0, NECGPU_K_TRSM));
        }
      }
      if (rest <= 0) continue;
      if (bulk_pending && panel_top) CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_bulk, 0));
      // trailing update with K = outer
      const int kk = (int)(KE - K0);
      if (la && rest > outer) {
        TRY(tc_pack<F>(e, 1, M + KE * ld + K0, M + K0 * ld + KE, ld, rest, rest, kk, !u12_emit));
        TRY(tc_run<F>(e, 1, rest, 0, outer, kk, M + KE * ld + KE, ld, e->stream, e->nsm));  // next outer block
        CUDA_TRY(cudaEventRecord(e->ev_fork, e->stream));
        CUDA_TRY(cudaStreamWaitEvent(e->stream2, e->ev_fork, 0));
        TRY(tc_run<F>(e, 1, rest, outer, rest - outer, kk, M + KE * ld + KE + outer, ld, e->stream2,
                   e->nsm - e->lookahead_sms));
        CUDA_TRY(cudaEventRecord(e->ev_far, e->stream2));
        far_pending = true;
      } else {
        TRY(gemm(KE, KE, K0, rest, rest, kk));
      }
    }
    if (far_pending) CUDA_TRY(cudaStreamWaitEvent(e->stream, e->ev_far, 0));
    return 0;
  };
  // operand buffers at their largest sizes before any capture (no
  // allocation happens inside the launches below)
  if (e->use_tc) {
    TRY(ensure_tc<F>(e, F::kKMul * (int)outer, n, 0));
    if (la) TRY(ensure_tc<F>(e, F::kKMul * (int)outer, n, 1));
    if (split_inner) {
      const size_t need = 2 * (size_t)e->tc_rows * (size_t)e->tc_kbytes;
      if (!e->d_Bp3 || e->bp3_bytes < need) {
        TRY(dalloc(e, e->d_Bp3, need));
        e->bp3_bytes = need;
      }
    }
  }
  // CUDA graph of the launch sequence: it depends only on the size, the
  // tuning and the buffers, so the second factorisation with the same ones
  // is captured and every later one replays the graph (no per-launch host
  // submission, shorter gaps between the dependent launches of the panel
  // chain).  Not while launches are timed, nor when the stream is the legacy
  // default stream or is being captured by the caller.
  LuGraphKey key{};
  key.n = n, key.ld = ld, key.outer = outer, key.la = la, key.la_sms = e->lookahead_sms;
  key.group = e->gemm_group, key.use_tc = e->use_tc + 2 * (int)F::kFormat;
  key.trsm8 = (e->l21_rows ? 64 : 0) + (panel_top ? 32 : 0) + (e->chain_prio ? 16 : 0) + e->trsm8 * 8 + (split_inner ? 4 : 0) +
              (u12_fused ? 2 : 0) + (fused_pack ? 1 : 0);
  key.nsm = e->nsm * 4096 + e->side_ctas;
  key.ptr[0] = M, key.ptr[1] = e->d_piv, key.ptr[2] = e->d_src, key.ptr[3] = e->d_dinv;
  key.ptr[4] = e->d_status, key.ptr[5] = e->d_Ap, key.ptr[6] = e->d_Bp, key.ptr[7] = e->d_Ap2;
  key.ptr[8] = e->d_Bp2, key.ptr[9] = e->stream, key.ptr[10] = e->stream2, key.ptr[11] = e->stream3;
  key.ptr[12] = e->d_Bp3, key.ptr[13] = e->stream4, key.ptr[14] = e->d_top_cnt;
  key.ptr[15] = e->d_Bpan;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(e->stream, &cap));
  const bool graphs = e->lu_graphs && e->timing_level < 2 && e->stream && cap == cudaStreamCaptureStatusNone;
  if (graphs && e->lu_exec && e->lu_key == key) {
    CUDA_TRY(cudaGraphLaunch(e->lu_exec, e->stream));
    e->launches += e->lu_exec_launches;
  } else if (graphs && e->lu_seen == key) {
    if (e->lu_exec) {
      cudaGraphExecDestroy(e->lu_exec);
      e->lu_exec = nullptr;
    }
    const int64_t l0 = e->launches;
    CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    const int rc = issue();
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return rc ? rc : fail(e, NECGPU_ERR_CUDA, std::string("LU graph capture: ") + cudaGetErrorString(ce));
    }
    const cudaError_t ie = cudaGraphInstantiate(&e->lu_exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      e->lu_exec = nullptr;
      return fail(e, NECGPU_ERR_CUDA, std::string("LU graph instantiate: ") + cudaGetErrorString(ie));
    }
    e->lu_key = key;
    e->lu_exec_launches = e->launches - l0;
    CUDA_TRY(cudaGraphLaunch(e->lu_exec, e->stream));
  } else {
    TRY(issue());
    e->lu_seen = key;
  }
  std::vector<int> piv(n), perm(n);
  CUDA_TRY(cudaMemcpyAsync(piv.data(), e->d_piv, n * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += n * sizeof(int);
  int st = 0;
  TRY(sync_status(e, &st));
  for (int64_t i = 0; i < n; i++) perm[i] = (int)i;
  for (int64_t k = 0; k < n; k++) {
    int p = piv[k];
    if (p < 0 || p >= n) return fail(e, NECGPU_ERR_NONFINITE, "LU: invalid pivot index");
    std::swap(perm[k], perm[p]);
  }
  TRY(upload(e, e->d_perm, perm.data(), perm.size()));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (st & tc::kStatTimeout) return fail(e, NECGPU_ERR_CUDA, "LU: tensor-core update pipeline timed out");
  if (st & kLuStatNonFinite) return fail(e, NECGPU_ERR_NONFINITE, "LU: NaN/Inf in the matrix");
  if (st & kLuStatSingular) return fail(e, NECGPU_ERR_SINGULAR, "LU: zero pivot in a diagonal block");
  return 0;
}

// ---------------- triangular solves ----------------
// x (factor precision, in d_w1) = U^-1 L^-1 P b
template <typename R>
int run_trsv(necgpu_engine* e, const typename cvec<R>::T* M, typename cvec<R>::T* rhs,
             typename cvec<R>::T* sol) {
  using T = typename cvec<R>::T;
  const int64_t n = e->n, ld = e->ld;
  const int nblk = (int)((n + kTrsvB - 1) / kTrsvB);
  constexpr size_t dsm = trsv_diag_smem<T>();
  if (e->sweep_trsv) {
    // persistent sweeps: one cooperative launch per triangle
    if (!e->d_flags) {
      TRY(dalloc(e, e->d_flags, (size_t)nblk));
      CUDA_TRY(cudaMemsetAsync(e->d_flags, 0, nblk * sizeof(int), e->stream));
      e->flag_epoch = 0;
    }
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    int per_sm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_sweep_kernel<T, true>, kSweepThreads, dsm));
    const int grid = std::max(1, std::min(nblk, per_sm * e->nsm));
    const double tri_bytes = 0.5 * (double)n * (double)n * sizeof(T);
    for (int pass = 0; pass < 2; pass++) {
      int epoch = ++e->flag_epoch;
      const T* src = pass == 0 ? rhs : sol;
      T* dst = pass == 0 ? sol : rhs;
      void* args[] = {(void*)&M, (void*)&ld, (void*)&n, (void*)&src, (void*)&dst, (void*)&e->d_flags, (void*)&epoch,
                      (void*)&e->d_status};
      const int kt = kbegin(e);
      CUDA_TRY(cudaLaunchCooperativeKernel(pass == 0 ? (const void*)trsv_sweep_kernel<T, true>
                                                     : (const void*)trsv_sweep_kernel<T, false>,
                                           dim3(grid), dim3(kSweepThreads), args, dsm, e->stream));
      kend(e, kt, NECGPU_K_TRSV, tri_bytes, nullptr, "trsv_sweep_kernel");
      LAUNCHED();
    }
    // the backward pass wrote the solution into rhs; return it in sol
    CUDA_TRY(cudaMemcpyAsync(sol, rhs, n * sizeof(T), cudaMemcpyDeviceToDevice, e->stream));
    return 0;
  }
  CUDA_TRY(cudaFuncSetAttribute(trsv_diag_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
  CUDA_TRY(cudaFuncSetAttribute(trsv_diag_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
  // the 'flops' recorded for the solves are the bytes of factor read
  for (int k = 0; k < nblk; k++) {
    const int64_t b0 = (int64_t)k * kTrsvB;
    KLAUNCH(NECGPU_K_TRSV, (double)kTrsvB * kTrsvB * sizeof(T),
            trsv_diag_kernel<T, true><<<1, 64, dsm, e->stream>>>(M, ld, n, b0, rhs, sol));
    const int64_t r0 = b0 + kTrsvB;
    if (r0 < n) {
      unsigned g = (unsigned)std::min<int64_t>((n - r0 + 7) / 8, 4 * e->nsm);
      KLAUNCH(NECGPU_K_TRSV, (double)(n - r0) * kTrsvB * sizeof(T),
              trsv_update_kernel<T><<<g, 256, 0, e->stream>>>(M, ld, n, b0, r0, n, sol, rhs));
    }
  }
  // backward: sol holds y; reuse rhs as the running right-hand side
  CUDA_TRY(cudaMemcpyAsync(rhs, sol, n * sizeof(T), cudaMemcpyDeviceToDevice, e->stream));
  for (int k = nblk - 1; k >= 0; k--) {
    const int64_t b0 = (int64_t)k * kTrsvB;
    KLAUNCH(NECGPU_K_TRSV, (double)kTrsvB * kTrsvB * sizeof(T),
            trsv_diag_kernel<T, false><<<1, 64, dsm, e->stream>>>(M, ld, n, b0, rhs, sol));
    if (b0 > 0) {
      unsigned g = (unsigned)std::min<int64_t>((b0 + 7) / 8, 4 * e->nsm);
      KLAUNCH(NECGPU_K_TRSV, (double)b0 * kTrsvB * sizeof(T),
              trsv_update_kernel<T><<<g, 256, 0, e->stream>>>(M, ld, n, b0, 0, b0, sol, rhs));
    }
  }
  return 0;
}

int ensure_vectors(necgpu_engine* e) {
  const int64_t n = e->n;
  if (!e->d_b) TRY(dalloc(e, e->d_b, n));
  if (!e->d_x) TRY(dalloc(e, e->d_x, n));
  if (!e->d_r) TRY(dalloc(e, e->d_r, n));
  if (!e->d_cur) TRY(dalloc(e, e->d_cur, n));
  if (!e->d_w1) TRY(dalloc(e, e->d_w1, n));
  if (!e->d_w2) TRY(dalloc(e, e->d_w2, n));
  if (!e->d_abc) TRY(dalloc(e, e->d_abc, 6 * (size_t)n));
  if (!e->d_rn2) TRY(dalloc(e, e->d_rn2, 2));
  return 0;
}

// Inverses of the 64 x 64 diagonal blocks of the complex64 factors, for the
// refinement sweeps (one CTA per block, all blocks at once).
int invert_diag_blocks(necgpu_engine* e, bool force = false) {
  if (!e->inv_sweep && !force) return 0;
  const int64_t nblk = (e->n + kBlk - 1) / kBlk;
  if (!e->d_tinv) TRY(dalloc(e, e->d_tinv, (size_t)nblk * 2 * kBlk * kBlk));
  if (!e->d_sweep_ctr) TRY(dalloc(e, e->d_sweep_ctr, 4));
  CUDA_TRY(cudaFuncSetAttribute(tri_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_inv_smem()));
  KLAUNCH(NECGPU_K_OTHER, 0.0,
          tri_inv_kernel<<<(unsigned)nblk, 128, tri_inv_smem(), e->stream>>>(e->Z32, e->ld, e->n, e->d_tinv));
  if (!e->d_wnext) TRY(dalloc(e, e->d_wnext, (size_t)nblk * 2 * kSweepDepth * kBlk * kBlk));
  CUDA_TRY(cudaFuncSetAttribute(next_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)next_tile_smem()));
  KLAUNCH(NECGPU_K_OTHER, 0.0,
          next_tile_kernel<<<dim3((unsigned)nblk, 2, kSweepDepth), 256, next_tile_smem(), e->stream>>>(
              e->Z32, e->ld, e->n, e->d_tinv, e->d_wnext));
  return 0;
}

// sol = U^-1 L^-1 rhs on the complex64 factors with inverted diagonal
// blocks (rhs is overwritten): two persistent sweeps
int run_trsv_inv_on(necgpu_engine* e, const float2* Mf, const float2* tinv_blocks, const float2* wnext_blocks,
                    float2* rhs, float2* sol) {
  const int64_t n = e->n, ld = e->ld;
  const int nblk = (int)((n + kBlk - 1) / kBlk);
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, inv_sweep_kernel<true>, kInvSweepThreads, 0));
  if (per_sm < 1) return fail(e, NECGPU_ERR_CUDA, "sweep kernel cannot be resident");
  const int grid = std::max(1, std::min(nblk, per_sm * e->nsm));
  const double tri_bytes = 0.5 * (double)n * (double)n * sizeof(float2);
  // clusters of 16 (or 8) CTAs, one position each, when every cluster can be
  // resident at once (a cooperative launch)
  const int CS = e->sweep_cluster >= 16 ? 16 : 8;
  const int gridc = (nblk + CS - 1) / CS * CS;
  cudaLaunchConfig_t ccfg = {};
  cudaLaunchAttribute cattr[2];
  ccfg.gridDim = dim3((unsigned)gridc);
  ccfg.blockDim = dim3(kInvSweepThreads);
  ccfg.stream = e->stream;
  cattr[0].id = cudaLaunchAttributeClusterDimension;
  cattr[0].val.clusterDim.x = CS;
  cattr[0].val.clusterDim.y = 1;
  cattr[0].val.clusterDim.z = 1;
  cattr[1].id = cudaLaunchAttributeCooperative;
  cattr[1].val.cooperative = 1;
  ccfg.attrs = cattr;
  ccfg.numAttrs = 2;
  bool clustered = false;
  if (e->sweep_cluster) {
    int ncl = 0;
    ccfg.numAttrs = 1;  // the occupancy query takes the cluster shape only
    if (CS == 16) {
      for (auto* k : {inv_sweep_kernel<true, 16>, inv_sweep_kernel<false, 16>})
        if (cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) ncl = -1;
      clustered = ncl == 0 && cudaOccupancyMaxActiveClusters(&ncl, inv_sweep_kernel<true, 16>, &ccfg) == cudaSuccess &&
                  (int64_t)ncl * CS >= gridc;
    } else {
      clustered = cudaOccupancyMaxActiveClusters(&ncl, inv_sweep_kernel<true, 8>, &ccfg) == cudaSuccess &&
                  (int64_t)ncl * CS >= gridc;
    }
    ccfg.numAttrs = 2;
    if (!clustered) {
      (void)cudaGetLastError();
      e->sweep_cluster = CS == 16 ? 8 : 0;  // the next solve tries eight, then none
    }
  }
  for (int pass = 0; pass < 2; pass++) {
    const float2* src = pass == 0 ? rhs : sol;
    float2* dst = pass == 0 ? sol : rhs;
    const float2* tinv = tinv_blocks;
    const float2* wnext = wnext_blocks;
    unsigned* counter = e->d_sweep_ctr;
    CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), e->stream));
    // every element of the solution starts as the sweep's unset marker
    // (kSweepUnset in both halves), polled by the block after its owner
    CUDA_TRY(cudaMemsetAsync(dst, 0xFF, n * sizeof(float2), e->stream));
    void* args[] = {(void*)&Mf,  (void*)&ld,  (void*)&n,       (void*)&tinv,       (void*)&wnext,
                    (void*)&src, (void*)&dst, (void*)&counter, (void*)&e->d_status};
    const int kt = kbegin(e);
    if (clustered) {
      const cudaError_t le =
          CS == 16 ? cudaLaunchKernelEx(&ccfg, pass == 0 ? inv_sweep_kernel<true, 16> : inv_sweep_kernel<false, 16>, Mf,
                                        ld, n, tinv, wnext, src, dst, counter, e->d_status)
                   : cudaLaunchKernelEx(&ccfg, pass == 0 ? inv_sweep_kernel<true, 8> : inv_sweep_kernel<false, 8>, Mf, ld,
                                        n, tinv, wnext, src, dst, counter, e->d_status);
      if (le != cudaSuccess) {  // the configuration was refused: the launch below instead, from now on
        (void)cudaGetLastError();
        clustered = false;
        e->sweep_cluster = 0;
      }
    }
    if (!clustered)
      CUDA_TRY(cudaLaunchCooperativeKernel(pass == 0 ? (const void*)inv_sweep_kernel<true>
                                                     : (const void*)inv_sweep_kernel<false>,
                                           dim3(grid), dim3(kInvSweepThreads), args, 0, e->stream));
    kend(e, kt, NECGPU_K_TRSV, tri_bytes, nullptr, clustered ? "inv_sweep_kernel (clusters)" : "inv_sweep_kernel");
    LAUNCHED();
  }
  // the backward pass wrote the solution into rhs
  CUDA_TRY(cudaMemcpyAsync(sol, rhs, n * sizeof(float2), cudaMemcpyDeviceToDevice, e->stream));
  return 0;
}
int run_trsv_inv(necgpu_engine* e, float2* rhs, float2* sol) {
  return run_trsv_inv_on(e, e->Z32, e->d_tinv, e->d_wnext, rhs, sol);
}

// Mixed-precision factorisation of the FP64 matrix: demote to complex64, then
// LU with block-local pivoting (blockpiv) or full partial pivoting.
// Operand format of the next mixed factorisation.  TF32 saves a third of the
// update's tensor-core time (~2 ms at 11,520 unknowns, growing as n^3) and
// costs a refinement step or more (~1.2 ms there, growing as n to n^2), so
// it is taken only for large systems, and no longer once a TF32
// factorisation of this engine needed many refinement steps (a badly
// conditioned structure, whose next frequencies would do the same).
int pick_format(const necgpu_engine* e) {
  if (e->tc_format) return e->tc_format;
  return e->n >= e->tf32_min_n && !e->tf32_demoted ? 2 : 1;
}

int factor_mixed(necgpu_engine* e, bool blockpiv) {
  if (!e->Z32) TRY(dalloc(e, e->Z32, (size_t)e->n * e->ld));
  if (!e->z32_fresh)
    KLAUNCH(NECGPU_K_OTHER, 0.0, demote_kernel<<<8 * e->nsm, 256, 0, e->stream>>>(e->Z64, e->Z32, e->n * e->ld));
  e->z32_fresh = false;  // the factorisation overwrites it
  e->blockpiv = blockpiv;
  e->stats.pivoting = blockpiv ? 1 : 0;
  e->adj_ready = false;
  const int fmt = pick_format(e);
  e->tc_format_used = fmt;
  if (blockpiv) {
    const int rc = fmt == 2 ? run_lu_blockpiv<tc::Tf32>(e, e->Z32) : run_lu_blockpiv<tc::SplitBf16>(e, e->Z32);
    if (rc != NECGPU_ERR_SINGULAR && rc != NECGPU_ERR_NONFINITE) return rc ? rc : invert_diag_blocks(e);
    // a diagonal block without a usable pivot: full partial pivoting
    CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
    return factor_mixed(e, false);
  }
  TRY((fmt == 2 ? run_lu<float, tc::Tf32>(e, e->Z32) : run_lu<float>(e, e->Z32)));
  return invert_diag_blocks(e);
}

// Iterative refinement with the complex64 factors against the FP64 matrix:
// x = 0, r = b; repeat d = LU^-1 r, x += d, r = b - Z x (FP64) until the
// relative residual reaches the tolerance or stops decreasing.
int refine(necgpu_engine* e, int* iters, double* rel_out) {
  const int64_t n = e->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  float2* w1 = reinterpret_cast<float2*>(e->d_w1);
  float2* w2 = reinterpret_cast<float2*>(e->d_w2);
  CUDA_TRY(cudaMemsetAsync(e->d_x, 0, n * sizeof(double2), e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_r, e->d_b, n * sizeof(double2), cudaMemcpyDeviceToDevice, e->stream));
  const unsigned gr = (unsigned)std::min<int64_t>((n + 7) / 8, 8 * e->nsm);
  CUDA_TRY(cudaMemsetAsync(e->d_rn2, 0, 2 * sizeof(double), e->stream));
  KLAUNCH(NECGPU_K_OTHER, 0.0, norm2_kernel<<<g1, 256, 0, e->stream>>>(e->d_b, n, e->d_rn2 + 1));
  double prev = 1e300, rel = 1.0;
  int it = 0;
  for (; it <= e->refine_max; it++) {
    KLAUNCH(NECGPU_K_OTHER, 0.0, permute_kernel<float2, double2><<<g1, 256, 0, e->stream>>>(e->d_r, e->d_perm, w1, n));
    if (e->inv_sweep && e->sweep_trsv)
      TRY(run_trsv_inv(e, w1, w2));
    else
      TRY(run_trsv<float>(e, e->Z32, w1, w2));
    KLAUNCH(NECGPU_K_OTHER, 0.0, axpy_kernel<float2><<<g1, 256, 0, e->stream>>>(e->d_x, w2, n));
    CUDA_TRY(cudaMemsetAsync(e->d_rn2, 0, sizeof(double), e->stream));
    // bytes of FP64 Z read by the residual
    KLAUNCH(NECGPU_K_RESID, (double)n * n * sizeof(double2),
            residual_kernel<<<gr, 256, 0, e->stream>>>(e->Z64, e->ld, n, e->d_x, e->d_b, e->d_r, e->d_rn2));
    double rn2[2] = {0, 0};
    int st = 0;
    CUDA_TRY(cudaMemcpyAsync(rn2, e->d_rn2, 2 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaMemcpyAsync(&st, e->d_status, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    e->stats.d2h_bytes += 2 * sizeof(double) + sizeof(int);
    kflush(e);
    if (st & (1 << 9)) return fail(e, NECGPU_ERR_CUDA, "refinement: triangular sweep gave up waiting on a block");
    const double bn = std::sqrt(rn2[1]);
    rel = bn > 0 ? std::sqrt(rn2[0]) / bn : 0.0;
    if (!std::isfinite(rel)) {
      *iters = it + 1;
      *rel_out = rel;
      return fail(e, NECGPU_ERR_NONFINITE, "refinement: non-finite residual");
    }
    if (rel <= e->refine_tol || rel > 0.5 * prev) {  // converged, or at the FP64 floor
      it++;
      break;
    }
    prev = rel;
  }
  *iters = it;
  *rel_out = rel;
  return 0;
}

// ---------------- adjoint solves ----------------
// Transposed copies of the held mixed factors, of the FP64 matrix and of the
// inverted diagonal blocks (once per factorisation).
int ensure_adjoint(necgpu_engine* e) {
  if (e->factored != NECGPU_MIXED)
    return fail(e, NECGPU_ERR_UNSUPPORTED,
                "adjoint: needs the mixed-precision factorisation (the FP64 path factors Z in place)");
  if (e->adj_ready) return 0;
  const int64_t n = e->n, ld = e->ld, nblk = (n + kBlk - 1) / kBlk;
  if (!e->inv_sweep || !e->d_tinv) TRY(invert_diag_blocks(e, true));
  if (!e->ZT32) TRY(dalloc(e, e->ZT32, (size_t)n * ld));
  if (!e->ZT64) TRY(dalloc(e, e->ZT64, (size_t)n * ld));
  if (!e->d_tinvT) TRY(dalloc(e, e->d_tinvT, (size_t)nblk * 2 * kBlk * kBlk));
  const dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  KLAUNCH(NECGPU_K_OTHER, 0.0, transpose_kernel<float2><<<g, 256, 0, e->stream>>>(e->Z32, ld, e->ZT32, ld, n));
  KLAUNCH(NECGPU_K_OTHER, 0.0, transpose_kernel<double2><<<g, 256, 0, e->stream>>>(e->Z64, ld, e->ZT64, ld, n));
  KLAUNCH(NECGPU_K_OTHER, 0.0, tinv_transpose_kernel<<<(unsigned)nblk, 256, 0, e->stream>>>(e->d_tinv, e->d_tinvT));
  if (!e->d_wnextT) TRY(dalloc(e, e->d_wnextT, (size_t)nblk * 2 * kSweepDepth * kBlk * kBlk));
  CUDA_TRY(cudaFuncSetAttribute(next_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)next_tile_smem()));
  KLAUNCH(NECGPU_K_OTHER, 0.0,
          next_tile_kernel<<<dim3((unsigned)nblk, 2, kSweepDepth), 256, next_tile_smem(), e->stream>>>(
              e->ZT32, ld, n, e->d_tinvT, e->d_wnextT));
  e->adj_ready = true;
  return 0;
}

// Z^T w = phi (device vectors), refined in FP64 against Z^T like the forward
// solve: w = 0, r = phi; repeat d = P^T L^-T U^-T r, w += d, r = phi - Z^T w.
int refine_T(necgpu_engine* e, const double2* phi, double2* w, int* iters, double* rel_out) {
  const int64_t n = e->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  float2* w1 = reinterpret_cast<float2*>(e->d_w1);
  float2* w2 = reinterpret_cast<float2*>(e->d_w2);
  double2* r = e->d_adj_r;
  CUDA_TRY(cudaMemsetAsync(w, 0, n * sizeof(double2), e->stream));
  CUDA_TRY(cudaMemcpyAsync(r, phi, n * sizeof(double2), cudaMemcpyDeviceToDevice, e->stream));
  const unsigned gr = (unsigned)std::min<int64_t>((n + 7) / 8, 8 * e->nsm);
  CUDA_TRY(cudaMemsetAsync(e->d_rn2, 0, 2 * sizeof(double), e->stream));
  KLAUNCH(NECGPU_K_OTHER, 0.0, norm2_kernel<<<g1, 256, 0, e->stream>>>(phi, n, e->d_rn2 + 1));
  double prev = 1e300, rel = 1.0;
  int it = 0;
  for (; it <= e->refine_max; it++) {
    KLAUNCH(NECGPU_K_OTHER, 0.0, demote_kernel<<<g1, 256, 0, e->stream>>>(r, w1, n));
    TRY(run_trsv_inv_on(e, e->ZT32, e->d_tinvT, e->d_wnextT, w1, w2));
    KLAUNCH(NECGPU_K_OTHER, 0.0, axpy_scatter_kernel<<<g1, 256, 0, e->stream>>>(w, w2, e->d_perm, n));
    CUDA_TRY(cudaMemsetAsync(e->d_rn2, 0, sizeof(double), e->stream));
    KLAUNCH(NECGPU_K_RESID, (double)n * n * sizeof(double2),
            residual_kernel<<<gr, 256, 0, e->stream>>>(e->ZT64, e->ld, n, w, phi, r, e->d_rn2));
    double rn2[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(rn2, e->d_rn2, 2 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    e->stats.d2h_bytes += 2 * sizeof(double);
    kflush(e);
    const double bn = std::sqrt(rn2[1]);
    rel = bn > 0 ? std::sqrt(rn2[0]) / bn : 0.0;
    if (!std::isfinite(rel)) {
      *iters = it + 1;
      *rel_out = rel;
      return fail(e, NECGPU_ERR_NONFINITE, "adjoint: non-finite residual");
    }
    if (rel <= e->refine_tol || rel > 0.5 * prev) {
      it++;
      break;
    }
    prev = rel;
  }
  *iters = it;
  *rel_out = rel;
  return 0;
}

FarDir engine_far_dir(const necgpu_engine* e, double theta, double phi) {
  return far_dir(theta, phi, e->ground == kGroundNone ? 1 : 2, e->ground == kGroundPerfect ? 1 : 0, e->P.zrati,
                 e->P.eta);
}

// Solve Z x = b (d_b) into d_x (FP64) with the held factors; then the
// current coefficients into d_abc / d_cur.
int run_solve(necgpu_engine* e, bool sync_checks) {
  const int64_t n = e->n;
  const unsigned g1 = (unsigned)((n + 255) / 256);
  e->stats.refine_iters = 0;
  e->stats.refine_residual = 0.0;
  if (e->factored == NECGPU_FP64) {
    KLAUNCH(NECGPU_K_OTHER, 0.0,
            permute_kernel<double2, double2><<<g1, 256, 0, e->stream>>>(e->d_b, e->d_perm, e->d_w1, n));
    TRY(run_trsv<double>(e, e->Z64, e->d_w1, e->d_x));
  } else if (e->factored == NECGPU_MIXED) {
    int it = 0;
    double rel = 1.0;
    int rc = refine(e, &it, &rel);
    const bool tf32 = e->tc_format_used == 2;
    if (!rc && tf32 && it > e->tf32_max_iters) e->tf32_demoted = true;
    if ((rc == NECGPU_ERR_NONFINITE || rel > kRefineFallback) && (e->blockpiv || (tf32 && e->tc_format == 0))) {
      // block-local pivoting (or the TF32 update) was not good enough for
      // this matrix: refactor the FP32 copy with full partial pivoting (and
      // split BF16 unless TF32 was asked for) and refine again
      if (tf32) e->tf32_demoted = true;
      TRY(factor_mixed(e, false));
      int it2 = 0;
      rc = refine(e, &it2, &rel);
      it += it2;
    }
    if (rc) return rc;
    e->stats.refine_iters = it;
    e->stats.refine_residual = rel;
    if (rel > 1e-6) return fail(e, NECGPU_ERR_REFINE, "refinement did not converge");
  } else {
    return fail(e, NECGPU_ERR_ARG, "solve: no factorisation held");
  }
  if (!e->matrix_only)
    KLAUNCH(NECGPU_K_OTHER, 0.0,
            coeff_kernel<<<g1, 256, 0, e->stream>>>(n, e->d_cptr, e->d_cbasis, e->d_ccoef, e->d_ccoef + e->nc,
                                                    e->d_ccoef + 2 * e->nc, e->d_x, e->d_abc, e->d_cur));
  if (sync_checks) CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->have_solution = true;
  return 0;
}

int run_pattern(necgpu_engine* e, int ndir) {
  PatternArgs a{};
  const int64_t n = e->n;
  a.n = n;
  a.ndir = ndir;
  a.theta = e->d_theta;
  a.phi = e->d_phi;
  a.x = e->d_seg;
  a.y = e->d_seg + n;
  a.z = e->d_seg + 2 * n;
  a.s = e->d_seg + 3 * n;
  a.cab = e->d_seg + 5 * n;
  a.sab = e->d_seg + 6 * n;
  a.salp = e->d_seg + 7 * n;
  a.abc = e->d_abc;
  a.ksymp = (e->ground == kGroundNone) ? 1 : 2;
  a.perfect = (e->ground == kGroundPerfect) ? 1 : 0;
  a.zrati = e->P.zrati;
  a.eta = e->P.eta;
  a.eth = e->d_eth;
  a.eph = e->d_eph;
  // work units: one per (direction, segment, image) term
  KLAUNCH(NECGPU_K_PATTERN, (double)ndir * n * a.ksymp,
          pattern_kernel<<<(unsigned)((ndir + kPatDirs - 1) / kPatDirs), kPatDirs * 32, 0, e->stream>>>(a));
  return 0;
}

int ensure_pattern(necgpu_engine* e, int ndir) {
  if (ndir <= e->pat_cap) return 0;
  TRY(dalloc(e, e->d_theta, ndir));
  TRY(dalloc(e, e->d_phi, ndir));
  TRY(dalloc(e, e->d_eth, ndir));
  TRY(dalloc(e, e->d_eph, ndir));
  e->pat_cap = ndir;
  return 0;
}

// ---------------- tuning table ----------------
constexpr necgpu_tuning kDefaultTuning = {256, 48, 16};

struct TuningRow {
  int precision;
  int64_t nmax;
  necgpu_tuning t;
};

bool tuning_valid(const necgpu_tuning& t) {
  return t.outer >= 64 && t.outer <= 1024 && t.outer % 64 == 0 && t.lookahead_sms >= 0 && t.lookahead_sms < 128 &&
         t.gemm_group >= 1 && t.gemm_group <= 1024;
}

// "precision n_max outer lookahead_sms gemm_group [anything]" per line; '#'
// starts a comment line.  False when the file cannot be read or a row is
// malformed.
bool parse_tuning(const char* path, std::vector<TuningRow>& rows) {
  FILE* f = std::fopen(path, "r");
  if (!f) return false;
  char line[512];
  bool ok = true;
  while (std::fgets(line, sizeof line, f)) {
    const char* p = line;
    while (*p == ' ' || *p == '\t') p++;
    if (*p == '#' || *p == '\n' || *p == '\r' || *p == 0) continue;
    char prec[16] = {0};
    long long nmax = 0;
    necgpu_tuning t{};
    if (std::sscanf(p, "%15s %lld %d %d %d", prec, &nmax, &t.outer, &t.lookahead_sms, &t.gemm_group) != 5) {
      ok = false;
      break;
    }
    const int pr = !std::strcmp(prec, "mixed") ? NECGPU_MIXED : !std::strcmp(prec, "fp64") ? NECGPU_FP64 : -1;
    if (pr < 0 || nmax < 1 || !tuning_valid(t)) {
      ok = false;
      break;
    }
    rows.push_back({pr, (int64_t)nmax, t});
  }
  std::fclose(f);
  return ok;
}

// The row for (precision, n): smallest n_max >= n, else the largest n_max.
bool tuning_row(const std::vector<TuningRow>& rows, int precision, int64_t n, necgpu_tuning* out) {
  const TuningRow* best = nullptr;
  const TuningRow* largest = nullptr;
  for (const TuningRow& r : rows) {
    if (r.precision != precision) continue;
    if (r.nmax >= n && (!best || r.nmax < best->nmax)) best = &r;
    if (!largest || r.nmax > largest->nmax) largest = &r;
  }
  if (!best) best = largest;
  if (!best) return false;
  *out = best->t;
  return true;
}

// Path of the library's table: NECPP_B200_TUNING, else tuning.tsv in the
// directory of the shared library holding this code ("" for none).
std::string library_tuning_path() {
  if (const char* s = std::getenv("NECPP_B200_TUNING")) return std::strcmp(s, "none") ? std::string(s) : "";
  Dl_info info;
  if (!dladdr(reinterpret_cast<const void*>(&library_tuning_path), &info) || !info.dli_fname) return "";
  std::string p(info.dli_fname);
  const size_t slash = p.rfind('/');
  return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tuning.tsv";
}

const std::vector<TuningRow>& library_tuning() {
  static std::vector<TuningRow> rows;
  static std::once_flag once;
  std::call_once(once, [] {
    const std::string path = library_tuning_path();
    if (path.empty() || !parse_tuning(path.c_str(), rows)) rows.clear();
  });
  return rows;
}

necgpu_tuning effective_tuning(const necgpu_engine* e, int precision, int64_t n) {
  necgpu_tuning t = kDefaultTuning;
  necgpu_tuning r;
  if (e->tuning_explicit)
    t = e->tuning_set;
  else if (tuning_row(library_tuning(), precision, n, &r))
    t = r;
  if (e->env_outer) t.outer = e->env_outer;
  if (e->env_lookahead_sms) t.lookahead_sms = e->env_lookahead_sms;
  if (e->env_lookahead == 0) t.lookahead_sms = 0;
  if (e->env_group) t.gemm_group = e->env_group;
  return t;
}

void select_tuning(necgpu_engine* e, int precision) {
  const necgpu_tuning t = effective_tuning(e, precision, e->n);
  e->outer = t.outer;
  e->lookahead = t.lookahead_sms > 0;
  if (t.lookahead_sms > 0) e->lookahead_sms = t.lookahead_sms;
  e->gemm_group = t.gemm_group;
}

int run_factor(necgpu_engine* e, int precision) {
  if (!e->filled) return fail(e, NECGPU_ERR_ARG, "factor: matrix not filled");
  select_tuning(e, precision);
  if (precision == NECGPU_FP64) {
    TRY(run_lu<double>(e, e->Z64));
    e->filled = false;  // Z64 now holds the factors
  } else if (precision == NECGPU_MIXED) {
    TRY(factor_mixed(e, e->prefer_blockpiv));
  } else {
    return fail(e, NECGPU_ERR_ARG, "factor: unknown precision");
  }
  e->factored = precision;
  e->adj_ready = false;
  return 0;
}

int fill_checked(necgpu_engine* e, bool want32) {
  // loads are applied to Z64 after the fill: their rows' copy would be stale
  want32 = want32 && !e->d_zload;
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  TRY(run_fill(e, true, want32));
  e->filled = true;
  e->factored = -1;
  e->z32_fresh = want32;
  return 0;
}

}  // namespace

// ======================= C-ABI =======================

namespace {

// Column-tile source lists of a structure's basis tables (fill.cuh): for
// every tile of kFillTB basis columns, the distinct contributing source
// segments (ascending) and their (column, a, b, c) entries.  ecoef = a | b | c.
// Built by a counting sort of the trio entries over tiles: each tile's
// entries keep the (source, entry) order of the trio tables.
struct TileLists {
  std::vector<int32_t> tile_ptr, tsrc, tsrc_eptr;
  std::vector<uint8_t> ecol;
  std::vector<double> ecoef;
};
void build_tile_lists(const necgpu_structure* s, int64_t n, int ntiles, TileLists& L) {
  const int32_t* tp = s->trio_ptr;
  const int64_t ne = tp[n];
  // entry k of the trio tables goes to position at[tile] of the tile-sorted order
  std::vector<int64_t> at(ntiles + 1, 0);
  for (int64_t k = 0; k < ne; k++) at[s->trio_basis[k] / kFillTB + 1]++;
  for (int t = 0; t < ntiles; t++) at[t + 1] += at[t];
  std::vector<int32_t> src(ne), ent(ne);  // per sorted position: source segment, trio entry
  {
    std::vector<int64_t> next(at.begin(), at.end() - 1);
    for (int64_t j = 0; j < n; j++)
      for (int32_t k = tp[j]; k < tp[j + 1]; k++) {
        const int64_t q = next[s->trio_basis[k] / kFillTB]++;
        src[q] = (int32_t)j;
        ent[q] = k;
      }
  }
  L.tile_ptr.assign(ntiles + 1, 0);
  L.tsrc.clear();
  L.tsrc_eptr.clear();
  L.tsrc.reserve(ne);
  L.tsrc_eptr.reserve(ne + 1);
  L.ecol.resize(ne);
  L.ecoef.assign(3 * std::max<int64_t>(ne, 1), 0.0);
  for (int t = 0; t < ntiles; t++) {
    L.tile_ptr[t] = (int32_t)L.tsrc.size();
    for (int64_t q = at[t]; q < at[t + 1]; q++) {
      if (q == at[t] || src[q] != src[q - 1]) {
        L.tsrc.push_back(src[q]);
        L.tsrc_eptr.push_back((int32_t)q);
      }
      const int32_t k = ent[q];
      L.ecol[q] = (uint8_t)(s->trio_basis[k] % kFillTB);
      L.ecoef[q] = s->trio_a[k];
      L.ecoef[ne + q] = s->trio_b[k];
      L.ecoef[2 * ne + q] = s->trio_c[k];
    }
  }
  L.tile_ptr[ntiles] = (int32_t)L.tsrc.size();
  L.tsrc_eptr.push_back((int32_t)ne);
}

// Per segment: the basis functions with support on it, ascending basis (the
// accumulation order of get_current_coefficients).  ccoef = a | b | c.
struct CoefLists {
  std::vector<int32_t> cptr, cbasis;
  std::vector<double> ccoef;
};
void build_coef_lists(const necgpu_structure* s, int64_t n, CoefLists& C) {
  const int32_t* tp = s->trio_ptr;
  const int64_t ntrio = tp[n];
  C.cptr.assign(n + 1, 0);
  C.cbasis.assign(std::max<int64_t>(ntrio, 1), 0);
  C.ccoef.assign(3 * std::max<int64_t>(ntrio, 1), 0.0);
  std::vector<int> order;
  for (int64_t j = 0; j < n; j++) {
    // a segment has a few entries: a stable insertion sort by basis
    order.clear();
    for (int32_t k = tp[j]; k < tp[j + 1]; k++) {
      size_t q = order.size();
      order.push_back(k);
      while (q > 0 && s->trio_basis[order[q - 1]] > s->trio_basis[k]) {
        order[q] = order[q - 1];
        q--;
      }
      order[q] = k;
    }
    C.cptr[j] = tp[j];
    for (size_t q = 0; q < order.size(); q++) {
      const int k = order[q];
      C.cbasis[tp[j] + q] = s->trio_basis[k];
      C.ccoef[tp[j] + q] = s->trio_a[k];
      C.ccoef[ntrio + tp[j] + q] = s->trio_b[k];
      C.ccoef[2 * ntrio + tp[j] + q] = s->trio_c[k];
    }
  }
  C.cptr[n] = tp[n];
}

}  // namespace

extern "C" {

int necgpu_create(necgpu_engine** out, int device) {
  if (!out) return NECGPU_ERR_ARG;
  auto* e = new necgpu_engine();
  *out = e;
  int count = 0;
  cudaError_t st = cudaGetDeviceCount(&count);
  if (st != cudaSuccess || count == 0)
    return fail(e, NECGPU_ERR_NO_DEVICE,
                std::string("no CUDA device: ") + (st != cudaSuccess ? cudaGetErrorString(st) : "count=0"));
  if (device < 0 || device >= count) return fail(e, NECGPU_ERR_ARG, "device index out of range");
  e->device = device;
  CUDA_TRY(cudaSetDevice(device));
  // three attributes instead of the whole property block (which costs
  // milliseconds per context)
  int major = 0, coop = 0, nsm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  if (major < 10) return fail(e, NECGPU_ERR_NO_DEVICE, "this build targets sm_100a (B200)");
  if (!coop) return fail(e, NECGPU_ERR_NO_DEVICE, "device lacks cooperative launch");
  e->nsm = nsm;
  if (const char* s = std::getenv("NECPP_B200_NO_TC")) e->use_tc = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_BLOCKED_TRSV")) e->sweep_trsv = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_PARTIAL_PIVOT")) e->prefer_blockpiv = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_FLAG_SWEEP")) e->inv_sweep = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_NO_DMMA")) e->use_dmma = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_LOOKAHEAD")) e->env_lookahead = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_TRSM1")) e->trsm8 = (s[0] == '0');
  if (const char* s = std::getenv("NECPP_B200_LU_GRAPH")) e->lu_graphs = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_U12_FUSED")) e->u12_fused = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_FUSED_PACK")) e->fused_pack = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_INNER_SPLIT")) e->inner_split = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_PANEL_TOP")) e->panel_top = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_SWEEP_CLUSTER")) {
    const int v = std::atoi(s);
    e->sweep_cluster = v >= 16 ? 16 : v >= 8 ? 8 : 0;
  }
  if (const char* s = std::getenv("NECPP_B200_L21_ROWS")) e->l21_rows = (s[0] != '0');
  if (const char* s = std::getenv("NECPP_B200_TC_FORMAT"))
    e->tc_format = !std::strcmp(s, "tf32") ? 2 : !std::strcmp(s, "bf16x3") ? 1 : 0;
  if (const char* s = std::getenv("NECPP_B200_TF32_MIN_N")) {
    const long long v = std::atoll(s);
    if (v >= 1) e->tf32_min_n = v;
  }
  if (const char* s = std::getenv("NECPP_B200_SIDE_CTAS")) {
    const int v = std::atoi(s);
    if (v >= 1 && v <= 1024) e->side_ctas = v;
  }
  {
    // the panel chain's launches take the device's greatest priority unless
    // NECPP_B200_PRIORITY=0
    int least = 0, greatest = 0;
    const char* s = std::getenv("NECPP_B200_PRIORITY");
    if ((!s || s[0] != '0') && cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess)
      e->chain_prio = greatest;
  }
  if (const char* s = std::getenv("NECPP_B200_GEMM_GROUP")) {
    const int v = std::atoi(s);
    if (v >= 1 && v <= 1024) e->env_group = v;
  }
  if (const char* s = std::getenv("NECPP_B200_LOOKAHEAD_SMS")) {
    const int v = std::atoi(s);
    if (v >= 1 && v < 128) e->env_lookahead_sms = v;
  }
  CUDA_TRY(cudaFuncSetAttribute(gemm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DmmaSmem)));
  if (const char* s = std::getenv("NECPP_B200_OUTER")) {
    const int64_t v = std::atoll(s);
    if (v >= 64 && v % 64 == 0 && v <= 1024) e->env_outer = (int)v;
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  e->own_stream = true;
  CUDA_TRY(cudaEventCreate(&e->ev0));
  CUDA_TRY(cudaEventCreate(&e->ev1));
  {
    // keep freed device memory in the default pool for reuse (process-local;
    // NECPP_B200_POOL_RELEASE=1 keeps the driver's default of releasing it)
    const char* rel = std::getenv("NECPP_B200_POOL_RELEASE");
    if (!(rel && rel[0] == '1')) {
      cudaMemPool_t pool;
      CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, device));
      uint64_t thr = UINT64_MAX;
      CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    }
  }
  TRY(dalloc(e, e->d_status, 4));
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  return NECGPU_OK;
}

int necgpu_destroy(necgpu_engine* e) {
  if (!e) return NECGPU_OK;
  if (e->stream) {
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
  }
  free_all(e);
  dfree(e, e->d_interp_carry);  // the interpolation cache lives as long as the engine
  dfree(e, e->d_status);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->stream2) {
    cudaStreamSynchronize(e->stream2);
    cudaStreamDestroy(e->stream2);
  }
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_far) cudaEventDestroy(e->ev_far);
  if (e->stream3) {
    cudaStreamSynchronize(e->stream3);
    cudaStreamDestroy(e->stream3);
  }
  if (e->ev_u12a) cudaEventDestroy(e->ev_u12a);
  if (e->ev_u12b) cudaEventDestroy(e->ev_u12b);
  if (e->stream4) {
    cudaStreamSynchronize(e->stream4);
    cudaStreamDestroy(e->stream4);
  }
  if (e->ev_diag) cudaEventDestroy(e->ev_diag);
  if (e->ev_bulk) cudaEventDestroy(e->ev_bulk);
  if (e->ev_swap) cudaEventDestroy(e->ev_swap);
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return NECGPU_OK;
}

const char* necgpu_last_error(const necgpu_engine* e) { return e ? e->err.c_str() : "null engine"; }

// One idle engine per device, kept between contexts: its streams, events,
// device buffers, tuned kernel attributes and captured LU graph serve the
// next structure of the same size without being built again.
namespace {
constexpr int kPoolDevices = 16;
std::mutex g_pool_mutex;
necgpu_engine* g_pool[kPoolDevices] = {};
}  // namespace

int necgpu_acquire(necgpu_engine** out, int device) {
  if (!out) return NECGPU_ERR_ARG;
  *out = nullptr;
  if (device >= 0 && device < kPoolDevices) {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (g_pool[device]) {
      *out = g_pool[device];
      g_pool[device] = nullptr;
      return NECGPU_OK;
    }
  }
  return necgpu_create(out, device);
}

int necgpu_release(necgpu_engine* e) {
  if (!e) return NECGPU_OK;
  if (e->touched || e->device < 0 || e->device >= kPoolDevices || cudaSetDevice(e->device) != cudaSuccess ||
      cudaStreamSynchronize(e->stream) != cudaSuccess)
    return necgpu_destroy(e);
  // forget what belonged to the context: its factors, solution, tables, the
  // interpolation cache's state and the engine-life format choice; keep the
  // buffers (the captured LU graph refers to them)
  e->factored = -1;
  e->have_solution = false;
  e->filled = false;
  e->somm_ready = false;
  e->adj_ready = false;
  e->tf32_demoted = false;
  e->interp_key = InterpKey{kInterpFresh, 0, 0, 0};
  e->stats = necgpu_stats{};
  e->launches = 0;
  e->err.clear();
  {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool[e->device]) {
      g_pool[e->device] = e;
      return NECGPU_OK;
    }
  }
  return necgpu_destroy(e);
}

int necgpu_set_stream(necgpu_engine* e, void* stream) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  CUDA_TRY(cudaSetDevice(e->device));
  if (e->stream) CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (stream == nullptr) {
    if (!e->own_stream) {
      CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
      e->own_stream = true;
    }
    return NECGPU_OK;
  }
  if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
  e->stream = (cudaStream_t)stream;
  e->own_stream = false;
  return NECGPU_OK;
}

int necgpu_enable_timing(necgpu_engine* e, int on) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  e->timing = on != 0;
  e->timing_level = on;
  return NECGPU_OK;
}

int necgpu_get_trace(necgpu_engine* e, necgpu_trace_rec* out, int cap) {
  if (!e || cap < 0) return -NECGPU_ERR_ARG;
  const int cnt = (int)std::min<size_t>(e->trace.size(), (size_t)cap);
  if (out) std::copy(e->trace.begin(), e->trace.begin() + cnt, out);
  return (int)e->trace.size();
}

int necgpu_reset_kernel_stats(necgpu_engine* e) {
  if (!e) return NECGPU_ERR_ARG;
  e->trace.clear();
  e->trace_based = false;
  for (int k = 0; k < NECGPU_K_COUNT; k++) {
    e->stats.k_ms[k] = 0;
    e->stats.k_launches[k] = 0;
    e->stats.k_flops[k] = 0;
  }
  return NECGPU_OK;
}

int necgpu_reuse_last_inputs(necgpu_engine* e) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (!e->last_rhs) return fail(e, NECGPU_ERR_ARG, "reuse_last_inputs: no solve has run");
  e->res_rhs = true;
  e->res_ndir = e->last_ndir;
  return NECGPU_OK;
}

int necgpu_set_refinement(necgpu_engine* e, double tol, int max_iter) {
  if (!e || !(tol > 0) || max_iter < 0) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  e->refine_tol = tol;
  e->refine_max = max_iter;
  return NECGPU_OK;
}

int necgpu_set_pivoting(necgpu_engine* e, int mode) {
  if (!e || (mode != 0 && mode != 1)) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  e->prefer_blockpiv = (mode == 1);
  return NECGPU_OK;
}

int necgpu_set_update_format(necgpu_engine* e, int format) {
  if (!e || format < 0 || format > 2) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  e->tc_format = format;
  e->tf32_demoted = false;
  return NECGPU_OK;
}

int necgpu_update_format(const necgpu_engine* e) {
  if (!e) return NECGPU_ERR_ARG;
  return e->factored == NECGPU_MIXED ? e->tc_format_used : 0;
}

int necgpu_get_stats(const necgpu_engine* e, necgpu_stats* out) {
  if (!e || !out) return NECGPU_ERR_ARG;
  *out = e->stats;
  out->launches = e->launches;
  return NECGPU_OK;
}

int necgpu_set_structure(necgpu_engine* e, const necgpu_structure* s) {
  if (!e) return NECGPU_ERR_ARG;
  if (!s || s->n < 2) return fail(e, NECGPU_ERR_ARG, "set_structure: need at least 2 segments");
  CUDA_TRY(cudaSetDevice(e->device));
  const int64_t n = s->n;
  if (n > (int64_t)1 << 28) return fail(e, NECGPU_ERR_ARG, "set_structure: too many segments");
  if (s->ground < 0 || s->ground > 3) return fail(e, NECGPU_ERR_ARG, "set_structure: bad ground type");
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (n != e->n) free_all(e);
  e->n = n;
  e->ld = (n + 63) / 64 * 64;  // 512 B-aligned FP32 rows: TMA bases of every 64-block sub-matrix
  e->ground = s->ground;
  e->use_exk = s->use_exk;
  e->P.rkh = s->rkh;
  e->P.eta = s->eta;
  e->P.zrati = mk(s->zrati_re, s->zrati_im);
  e->P.frati = mk(s->frati_re, s->frati_im);
  e->P.u = e->P.zrati;
  e->P.u2 = e->P.zrati * e->P.zrati;
  e->factored = -1;
  e->filled = false;
  e->have_solution = false;
  e->adj_ready = false;
  e->matrix_only = false;
  e->z32_fresh = false;
  dfree(e, e->d_zload);  // loads belong to one structure: set them after it
  e->somm_ready = false;   // so do the Sommerfeld tables (they follow the frequency)
  dfree(e, e->Z32);  // re-derived from Z64 when a mixed factorisation is asked for

  std::vector<double> seg(8 * n);
  for (int64_t i = 0; i < n; i++) {
    seg[i] = s->x[i];
    seg[n + i] = s->y[i];
    seg[2 * n + i] = s->z[i];
    seg[3 * n + i] = s->length[i];
    seg[4 * n + i] = s->radius[i];
    seg[5 * n + i] = s->cab[i];
    seg[6 * n + i] = s->sab[i];
    seg[7 * n + i] = s->salp[i];
  }
  std::vector<int32_t> ind(2 * n, 0);
  if (s->ek_ind1 && s->ek_ind2)
    for (int64_t i = 0; i < n; i++) {
      ind[i] = s->ek_ind1[i];
      ind[n + i] = s->ek_ind2[i];
    }

  const int32_t* tp = s->trio_ptr;
  if (tp[0] != 0) return fail(e, NECGPU_ERR_ARG, "set_structure: trio_ptr[0] != 0");
  for (int64_t j = 0; j < n; j++)
    if (tp[j + 1] < tp[j]) return fail(e, NECGPU_ERR_ARG, "set_structure: trio_ptr not ascending");
  const int64_t ntrio = tp[n];
  for (int64_t k = 0; k < ntrio; k++)
    if (s->trio_basis[k] < 0 || s->trio_basis[k] >= n)
      return fail(e, NECGPU_ERR_ARG, "set_structure: basis index out of range");

  const int ntiles = (int)((n + kFillTB - 1) / kFillTB);
  e->ntiles = ntiles;
  TileLists TL;
  build_tile_lists(s, n, ntiles, TL);
  const std::vector<int32_t>& tile_ptr = TL.tile_ptr;
  const std::vector<int32_t>& tsrc = TL.tsrc;
  const std::vector<int32_t>& tsrc_eptr = TL.tsrc_eptr;
  const std::vector<uint8_t>& ecol = TL.ecol;
  e->ne = (int64_t)ecol.size();
  const std::vector<double>& ecoef = TL.ecoef;
  CoefLists CL;
  build_coef_lists(s, n, CL);
  e->nc = ntrio;
  const std::vector<int32_t>& cptr = CL.cptr;
  const std::vector<int32_t>& cbasis = CL.cbasis;
  const std::vector<double>& ccoef = CL.ccoef;
  // kept to check perturbed structures (adjoint gradients) against this one
  e->h_tptr.assign(tp, tp + n + 1);
  e->h_tbasis.assign(s->trio_basis, s->trio_basis + ntrio);
  e->h_ind = ind;

  TRY(upload(e, e->d_seg, seg.data(), seg.size()));
  TRY(upload(e, e->d_ind, ind.data(), ind.size()));
  TRY(upload(e, e->d_tile_ptr, tile_ptr.data(), tile_ptr.size()));
  TRY(upload(e, e->d_tsrc, tsrc.data(), std::max<size_t>(tsrc.size(), 1)));
  TRY(upload(e, e->d_tsrc_eptr, tsrc_eptr.data(), tsrc_eptr.size()));
  TRY(upload(e, e->d_ecol, ecol.data(), std::max<size_t>(ecol.size(), 1)));
  TRY(upload(e, e->d_ecoef, ecoef.data(), ecoef.size()));
  TRY(upload(e, e->d_cptr, cptr.data(), cptr.size()));
  TRY(upload(e, e->d_cbasis, cbasis.data(), cbasis.size()));
  TRY(upload(e, e->d_ccoef, ccoef.data(), ccoef.size()));
  TRY(ensure_vectors(e));
  CUDA_TRY(cudaStreamSynchronize(e->stream));  // host staging freed on return
  return NECGPU_OK;
}

int necgpu_set_fill_precision(necgpu_engine* e, int precision) {
  if (!e) return NECGPU_ERR_ARG;
  if (precision != -1 && precision != NECGPU_FP64 && precision != NECGPU_MIXED)
    return fail(e, NECGPU_ERR_ARG, "set_fill_precision: -1, NECGPU_FP64 or NECGPU_MIXED");
  e->fill_precision = precision;
  return NECGPU_OK;
}

int necgpu_fill(necgpu_engine* e) {
  if (!e) return NECGPU_ERR_ARG;
  CUDA_TRY(cudaSetDevice(e->device));
  tick(e);
  TRY(fill_checked(e, e->fill_precision == NECGPU_MIXED));
  e->stats.ms_fill = tock(e);
  int st = 0;
  TRY(sync_status(e, &st));
  if (st & kStatSommerfeldTab)
    return fail(e, NECGPU_ERR_UNSUPPORTED,
                "fill: a segment pair lies within 0.95 wavelength of its ground image and no "
                "Sommerfeld tables are set (necgpu_set_sommerfeld)");
  if (st & kStatIterCap) return fail(e, NECGPU_ERR_NONFINITE, "fill: quadrature did not terminate (non-finite geometry?)");
  return NECGPU_OK;
}

int necgpu_factor(necgpu_engine* e, int precision) {
  if (!e) return NECGPU_ERR_ARG;
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  tick(e);
  TRY(run_factor(e, precision));
  e->stats.ms_factor = tock(e);
  return NECGPU_OK;
}

int necgpu_solve(necgpu_engine* e, const double* rhs, double* cur, double* abc) {
  if (!e || !rhs || !cur) return e ? fail(e, NECGPU_ERR_ARG, "solve: null argument") : NECGPU_ERR_ARG;
  CUDA_TRY(cudaSetDevice(e->device));
  const int64_t n = e->n;
  CUDA_TRY(cudaMemcpyAsync(e->d_b, rhs, n * sizeof(double2), cudaMemcpyHostToDevice, e->stream));
  e->stats.h2d_bytes += n * sizeof(double2);
  e->last_rhs = true;
  tick(e);
  TRY(run_solve(e, false));
  e->stats.ms_solve = tock(e);
  CUDA_TRY(cudaMemcpyAsync(cur, e->d_cur, n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += n * sizeof(double2);
  if (abc) {
    CUDA_TRY(cudaMemcpyAsync(abc, e->d_abc, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    e->stats.d2h_bytes += 6 * n * sizeof(double);
  }
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  kflush(e);
  for (int64_t i = 0; i < 2 * n; i++)
    if (!std::isfinite(cur[i])) return fail(e, NECGPU_ERR_NONFINITE, "solve: non-finite current");
  return NECGPU_OK;
}

int necgpu_pattern(necgpu_engine* e, int ndir, const double* theta, const double* phi, double* eth,
                   double* eph) {
  if (!e) return NECGPU_ERR_ARG;
  if (ndir <= 0 || !theta || !phi || !eth || !eph) return fail(e, NECGPU_ERR_ARG, "pattern: bad arguments");
  if (!e->have_solution) return fail(e, NECGPU_ERR_ARG, "pattern: no solution");
  CUDA_TRY(cudaSetDevice(e->device));
  TRY(ensure_pattern(e, ndir));
  CUDA_TRY(cudaMemcpyAsync(e->d_theta, theta, ndir * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_phi, phi, ndir * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  e->stats.h2d_bytes += 2 * ndir * sizeof(double);
  tick(e);
  TRY(run_pattern(e, ndir));
  e->stats.ms_pattern = tock(e);
  CUDA_TRY(cudaMemcpyAsync(eth, e->d_eth, ndir * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaMemcpyAsync(eph, e->d_eph, ndir * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += 2 * ndir * sizeof(double2);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  kflush(e);
  e->last_ndir = ndir;
  if (e->res_ndir > 0) e->res_ndir = ndir;  // the resident direction list was overwritten
  return NECGPU_OK;
}

int necgpu_device_z(necgpu_engine* e, void** z, int64_t* ld) {
  if (!e || !z || !ld) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  *z = e->Z64;
  *ld = e->ld;
  return NECGPU_OK;
}

int necgpu_copy_z(necgpu_engine* e, double* out) {
  if (!e || !out) return NECGPU_ERR_ARG;
  if (!e->filled || !e->Z64) return fail(e, NECGPU_ERR_ARG, "copy_z: no unfactored matrix held");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemcpy2DAsync(out, (size_t)e->n * sizeof(double2), e->Z64, (size_t)e->ld * sizeof(double2),
                               (size_t)e->n * sizeof(double2), (size_t)e->n, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return NECGPU_OK;
}

int necgpu_set_resident(necgpu_engine* e, const double* rhs, int ndir, const double* theta,
                        const double* phi) {
  if (!e || !rhs || ndir < 0) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemcpyAsync(e->d_b, rhs, e->n * sizeof(double2), cudaMemcpyHostToDevice, e->stream));
  if (ndir > 0) {
    TRY(ensure_pattern(e, ndir));
    CUDA_TRY(cudaMemcpyAsync(e->d_theta, theta, ndir * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->d_phi, phi, ndir * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->res_ndir = ndir;
  e->res_rhs = true;
  return NECGPU_OK;
}

// One full pass on resident inputs: fill -> factor -> solve -> coefficients
// -> far field.  The only host interaction is the pivot download inside the
// factorisation and the refinement's residual norms (mixed precision).
int necgpu_step_resident(necgpu_engine* e, int precision) {
  if (!e || !e->res_rhs) return e ? fail(e, NECGPU_ERR_ARG, "step: no resident inputs") : NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  CUDA_TRY(cudaSetDevice(e->device));
  tick(e);
  TRY(fill_checked(e, precision == NECGPU_MIXED));
  e->stats.ms_fill = tock(e);
  tick(e);
  TRY(run_factor(e, precision));
  e->stats.ms_factor = tock(e);
  tick(e);
  TRY(run_solve(e, false));
  e->stats.ms_solve = tock(e);
  tick(e);
  if (e->res_ndir > 0) TRY(run_pattern(e, e->res_ndir));
  e->stats.ms_pattern = tock(e);
  int st = 0;
  TRY(sync_status(e, &st));
  if (st & (kStatSommerfeldTab | kStatIterCap)) return fail(e, NECGPU_ERR_UNSUPPORTED, "step: fill status");
  return NECGPU_OK;
}

int necgpu_check_tc_gemm(necgpu_engine* e, int m, int n, int kb, unsigned seed, double* max_abs_diff,
                         double* max_abs_ref) {
  if (!e || m < 1 || n < 1 || kb < 1 || kb > 1024 || !max_abs_diff || !max_abs_ref) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  CUDA_TRY(cudaSetDevice(e->device));
  // operands at a 64-aligned offset o: A = X[o.., 0..kb), B = X[0..kb, o..),
  // C = X[o.., o..); rows of ld (a multiple of 64) keep C 16-byte aligned
  const int64_t o = ((int64_t)kb + 63) / 64 * 64;
  const int64_t rows = o + m, ld = (o + n + 63) / 64 * 64;
  float2 *X = nullptr, *Y = nullptr;
  float* d = nullptr;
  TRY(dalloc(e, X, (size_t)rows * ld));
  int rc = dalloc(e, Y, (size_t)rows * ld);
  if (!rc) rc = dalloc(e, d, 2);
  if (!rc) {
    const int64_t cnt = rows * ld;
    fill_random_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, e->stream>>>(X, cnt, seed);
    cudaMemcpyAsync(Y, X, cnt * sizeof(float2), cudaMemcpyDeviceToDevice, e->stream);
    cudaMemsetAsync(d, 0, 2 * sizeof(float), e->stream);
    cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream);
    // X: tensor cores; Y: CUDA-core FP32 reference of the same update
    rc = pick_format(e) == 2 ? tc_gemm_sub<tc::Tf32>(e, X + o * ld, X + o, X + o * ld + o, ld, m, n, kb)
                             : tc_gemm_sub<tc::SplitBf16>(e, X + o * ld, X + o, X + o * ld + o, ld, m, n, kb);
    if (!rc) {
      dim3 g((unsigned)((n + 63) / 64), (unsigned)((m + 63) / 64));
      gemm_sub_kernel<float><<<g, 256, 0, e->stream>>>(Y + o * ld, ld, Y + o, ld, Y + o * ld + o, ld, m, n, kb);
      max_diff_kernel<<<256, 256, 0, e->stream>>>(X + o * ld + o, Y + o * ld + o, ld, m, n, d);
      float h[2] = {0, 0};
      int st = 0;
      cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, e->stream);
      rc = sync_status(e, &st);
      if (!rc && (st & tc::kStatTimeout)) rc = fail(e, NECGPU_ERR_CUDA, "tensor-core GEMM pipeline timed out");
      if (!rc) {
        cudaError_t ce = cudaGetLastError();
        if (ce != cudaSuccess) rc = fail(e, NECGPU_ERR_CUDA, cudaGetErrorString(ce));
      }
      *max_abs_diff = h[0];
      *max_abs_ref = h[1];
    }
  }
  dfree(e, X);
  dfree(e, Y);
  dfree(e, d);
  return rc;
}

// Componentwise backward error of the factors F of P A (L unit lower, U
// upper; P A row i = A row perm[i]): max over i, j of
// |(P A - L U)_ij| / sum_k |L_ik| |U_kj| (|.|: |re| + |im|), and max |A|.
__global__ void lu_residual_kernel(const float2* A, const float2* F, const int* perm, int64_t ld, int64_t n,
                                   float* out) {
  float mx = 0.f, ref = 0.f;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / n, j = e - i * n;
    const int64_t kend = i < j ? i : j;
    float sr = 0.f, si = 0.f, sa = 0.f;
    for (int64_t k = 0; k <= kend; k++) {
      const float2 l = k == i ? make_float2(1.f, 0.f) : F[i * ld + k];
      const float2 u = F[k * ld + j];
      sr += l.x * u.x - l.y * u.y;
      si += l.x * u.y + l.y * u.x;
      sa += (fabsf(l.x) + fabsf(l.y)) * (fabsf(u.x) + fabsf(u.y));
    }
    const float2 a = A[(int64_t)perm[i] * ld + j];
    const float d = fabsf(a.x - sr) + fabsf(a.y - si);
    if (sa > 0.f) mx = fmaxf(mx, d / sa);
    ref = fmaxf(ref, fabsf(a.x) + fabsf(a.y));
  }
  atomicMax((int*)out, __float_as_int(mx));
  atomicMax((int*)out + 1, __float_as_int(ref));
}

int necgpu_matrix_solve(necgpu_engine* e, int64_t n, const double* z, const double* b, int precision, double* x,
                        double* residual) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (!z || !b || !x || n < 1 || n > 65536) return fail(e, NECGPU_ERR_ARG, "matrix_solve: bad arguments");
  if (precision != NECGPU_FP64 && precision != NECGPU_MIXED)
    return fail(e, NECGPU_ERR_ARG, "matrix_solve: unknown precision");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  free_all(e);  // a structure held before is dropped
  e->n = n;
  e->ld = (n + 63) / 64 * 64;
  e->matrix_only = true;
  int rc = dalloc(e, e->Z64, (size_t)n * e->ld);
  if (!rc) rc = ensure_vectors(e);
  if (!rc) {
    if (cudaMemcpy2DAsync(e->Z64, e->ld * sizeof(double2), z, n * sizeof(double2), n * sizeof(double2), n,
                          cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
        cudaMemcpyAsync(e->d_b, b, n * sizeof(double2), cudaMemcpyHostToDevice, e->stream) != cudaSuccess ||
        cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream) != cudaSuccess)
      rc = fail(e, NECGPU_ERR_CUDA, "matrix_solve: upload failed");
    e->stats.h2d_bytes += (n * n + n) * sizeof(double2);
  }
  if (!rc) {
    e->filled = true;
    e->factored = -1;
    rc = run_factor(e, precision);
  }
  if (!rc) rc = run_solve(e, true);
  if (!rc) {
    if (cudaMemcpyAsync(x, e->d_x, n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess ||
        cudaStreamSynchronize(e->stream) != cudaSuccess)
      rc = fail(e, NECGPU_ERR_CUDA, "matrix_solve: download failed");
    e->stats.d2h_bytes += n * sizeof(double2);
    if (residual) *residual = e->stats.refine_residual;
    for (int64_t i = 0; !rc && i < 2 * n; i++)
      if (!std::isfinite(x[i])) rc = fail(e, NECGPU_ERR_NONFINITE, "matrix_solve: non-finite solution");
  }
  kflush(e);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  free_all(e);  // the engine holds no structure or matrix afterwards
  e->matrix_only = false;
  return rc;
}

int necgpu_set_tuning(necgpu_engine* e, const necgpu_tuning* t) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (!t) {
    e->tuning_explicit = false;
    return NECGPU_OK;
  }
  if (!tuning_valid(*t))
    return fail(e, NECGPU_ERR_ARG,
                "set_tuning: outer must be a multiple of 64 in [64, 1024], lookahead_sms in [0, 127], gemm_group "
                "in [1, 1024]");
  e->tuning_set = *t;
  e->tuning_explicit = true;
  return NECGPU_OK;
}

int necgpu_get_tuning(const necgpu_engine* e, int precision, int64_t n, necgpu_tuning* out) {
  if (!e || !out || (precision != NECGPU_FP64 && precision != NECGPU_MIXED) || n < 1) return NECGPU_ERR_ARG;
  *out = effective_tuning(e, precision, n);
  return NECGPU_OK;
}

int necgpu_tuning_lookup(const char* path, int precision, int64_t n, necgpu_tuning* out) {
  if (!out || (precision != NECGPU_FP64 && precision != NECGPU_MIXED) || n < 1) return NECGPU_ERR_ARG;
  *out = kDefaultTuning;
  std::vector<TuningRow> rows;
  const std::string p = path ? std::string(path) : library_tuning_path();
  if (p.empty() || !parse_tuning(p.c_str(), rows)) return NECGPU_ERR_ARG;
  return tuning_row(rows, precision, n, out) ? NECGPU_OK : NECGPU_ERR_ARG;
}

int necgpu_measure_peak(necgpu_engine* e, int kind, double* tflops) {
  if (!e || !tflops || kind < 0 || kind > 1) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  CUDA_TRY(cudaSetDevice(e->device));
  const int ctas = 4 * e->nsm;
  double* sink = nullptr;
  TRY(dalloc(e, sink, (size_t)ctas * peak::kThreads));
  // a few milliseconds per launch; the best of three timed launches after one warm-up
  const int iters = kind == 0 ? 65536 : 16384;
  const double flops = kind == 0 ? (double)ctas * peak::kThreads * iters * 2.0 * peak::kChains
                                 : (double)ctas * (peak::kThreads / 32) * iters * 4.0 * 512.0;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  int rc = 0;
  float best = 0.f;
  if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) rc = NECGPU_ERR_CUDA;
  for (int rep = 0; rep < 4 && !rc; rep++) {
    cudaEventRecord(t0, e->stream);
    if (kind == 0)
      peak::dfma_peak_kernel<<<ctas, peak::kThreads, 0, e->stream>>>(sink, iters);
    else
      peak::dmma_peak_kernel<<<ctas, peak::kThreads, 0, e->stream>>>(sink, iters);
    cudaEventRecord(t1, e->stream);
    const cudaError_t ce = cudaEventSynchronize(t1);
    if (ce != cudaSuccess) {
      rc = fail(e, NECGPU_ERR_CUDA, cudaGetErrorString(ce));
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (rep > 0 && (best == 0.f || ms < best)) best = ms;
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  dfree(e, sink);
  if (!rc) *tflops = flops / (best * 1e-3) / 1e12;
  return rc;
}

int necgpu_check_block_lu(necgpu_engine* e, int n, unsigned seed, double* backward_err, double* max_abs,
                          int* interchanges) {
  if (!e || n < 1 || n > 4096 || !backward_err || !max_abs || !interchanges) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (e->n > 0) return fail(e, NECGPU_ERR_ARG, "check_block_lu: needs an engine without a structure");
  CUDA_TRY(cudaSetDevice(e->device));
  // the factorisation runs on the engine's own buffers, as for a structure
  // of n unknowns; the engine is left without a structure afterwards
  e->n = n;
  e->ld = (n + 63) / 64 * 64;
  select_tuning(e, NECGPU_MIXED);
  const int64_t ld = e->ld, cnt = (int64_t)n * ld;
  float2* A = nullptr;
  float* d = nullptr;
  int rc = dalloc(e, e->Z32, (size_t)cnt);
  if (!rc) rc = dalloc(e, A, (size_t)cnt);
  if (!rc) rc = dalloc(e, d, 2);
  if (!rc) {
    fill_random_kernel<<<(unsigned)((cnt + 255) / 256), 256, 0, e->stream>>>(e->Z32, cnt, seed);
    cudaMemcpyAsync(A, e->Z32, cnt * sizeof(float2), cudaMemcpyDeviceToDevice, e->stream);
    cudaMemsetAsync(d, 0, 2 * sizeof(float), e->stream);
    cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream);
    e->tc_format_used = pick_format(e);
    rc = e->tc_format_used == 2 ? run_lu_blockpiv<tc::Tf32>(e, e->Z32) : run_lu_blockpiv<tc::SplitBf16>(e, e->Z32);
    if (!rc) {
      lu_residual_kernel<<<8 * e->nsm, 256, 0, e->stream>>>(A, e->Z32, e->d_perm, ld, n, d);
      float h[2] = {0, 0};
      std::vector<int> piv(n);
      cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, e->stream);
      cudaMemcpyAsync(piv.data(), e->d_piv, n * sizeof(int), cudaMemcpyDeviceToHost, e->stream);
      const cudaError_t ce = cudaStreamSynchronize(e->stream);
      if (ce != cudaSuccess) rc = fail(e, NECGPU_ERR_CUDA, cudaGetErrorString(ce));
      int moved = 0;
      for (int k = 0; k < n; k++) moved += piv[k] != k;
      *backward_err = h[0];
      *max_abs = h[1];
      *interchanges = moved;
    }
  }
  dfree(e, A);
  dfree(e, d);
  free_all(e);
  return rc;
}

int necgpu_set_loads(necgpu_engine* e, const double* zload) {
  if (!e) return NECGPU_ERR_ARG;
  if (e->n <= 0) return fail(e, NECGPU_ERR_ARG, "set_loads: no structure set");
  CUDA_TRY(cudaSetDevice(e->device));
  if (!zload) {
    dfree(e, e->d_zload);
    return NECGPU_OK;
  }
  TRY(upload(e, e->d_zload, reinterpret_cast<const double2*>(zload), (size_t)e->n));
  e->filled = false;
  return NECGPU_OK;
}

int necgpu_set_sommerfeld(necgpu_engine* e, double eps_re, double eps_im) {
  if (!e) return NECGPU_ERR_ARG;
  if (e->n <= 0) return fail(e, NECGPU_ERR_ARG, "set_sommerfeld: no structure set");
  if (e->ground != kGroundSommerfeld) return fail(e, NECGPU_ERR_ARG, "set_sommerfeld: the structure has no Sommerfeld ground");
  CUDA_TRY(cudaSetDevice(e->device));
  if (!e->d_somm) TRY(dalloc(e, e->d_somm, (size_t)kSommPoints));
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  const unsigned blocks = (unsigned)((kSommEvalPoints + 31) / 32);
  KLAUNCH(NECGPU_K_FILL, 0.0,
          somm_table_kernel<<<blocks, 32, 0, e->stream>>>(mk(eps_re, eps_im), e->P.eta, e->d_somm, e->d_status));
  int st = 0;
  TRY(sync_status(e, &st));
  if (st & kStatIterCap) return fail(e, NECGPU_ERR_NONFINITE, "set_sommerfeld: a Sommerfeld integral did not converge");
  e->somm_ready = true;
  e->filled = false;
  return NECGPU_OK;
}

// nefld / nhfld over a list of points (nfpat, src/nec_context.cpp:5068-5186).
int necgpu_near_field(necgpu_engine* e, int magnetic, int npts, const double* pts, double* fields) {
  if (!e || npts < 0 || (npts > 0 && (!pts || !fields))) return e ? fail(e, NECGPU_ERR_ARG, "near_field: bad argument") : NECGPU_ERR_ARG;
  if (!e->have_solution) return fail(e, NECGPU_ERR_ARG, "near_field: no solution held (solve first)");
  if (npts == 0) return NECGPU_OK;
  CUDA_TRY(cudaSetDevice(e->device));
  const int64_t n = e->n;
  double* d_pts = nullptr;
  double2* d_out = nullptr;
  double2* d_near = nullptr;
  double* d_ax = nullptr;
  NearRecord* d_rec = nullptr;
  InterpKey* d_entry = nullptr;
  int* d_units = nullptr;
  auto cleanup = [&]() {
    dfree(e, d_pts);
    dfree(e, d_out);
    dfree(e, d_near);
    dfree(e, d_ax);
    dfree(e, d_rec);
    dfree(e, d_entry);
    dfree(e, d_units);
  };
  int rc = 0;
  do {
    if ((rc = upload(e, d_pts, pts, 3 * (size_t)npts))) break;
    if ((rc = dalloc(e, d_out, 3 * (size_t)npts))) break;
    CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
    NearFieldArgs a{};
    a.n = n;
    a.x = e->d_seg;
    a.y = e->d_seg + n;
    a.z = e->d_seg + 2 * n;
    a.s = e->d_seg + 3 * n;
    a.b = e->d_seg + 4 * n;
    a.cab = e->d_seg + 5 * n;
    a.sab = e->d_seg + 6 * n;
    a.salp = e->d_seg + 7 * n;
    a.ind1 = e->d_ind;
    a.ind2 = e->d_ind + n;
    a.P = e->P;
    a.P.near_g = nullptr;
    a.ground = e->ground;
    a.abc = e->d_abc;
    a.npts = npts;
    a.pts = d_pts;
    a.out = d_out;
    a.near = nullptr;
    a.status = e->d_status;
    const unsigned blocks = (unsigned)((npts + kNearWarps - 1) / kNearWarps);
    const bool x = e->use_exk != 0;
    if (magnetic) {
      KLAUNCH(NECGPU_K_PATTERN, (double)npts * (double)n,
              near_h_kernel<<<blocks, 32 * kNearWarps, 0, e->stream>>>(a));
    } else {
      if (e->ground == kGroundSommerfeld && e->somm_ready) {
        if ((rc = dalloc(e, d_near, 3 * (size_t)npts))) break;
        if ((rc = dalloc(e, d_ax, (size_t)npts))) break;
        if ((rc = dalloc(e, d_rec, (size_t)npts))) break;
        KLAUNCH(NECGPU_K_PATTERN, 0.0, near_radius_kernel<<<blocks, 32 * kNearWarps, 0, e->stream>>>(a, d_ax));
        auto launch = [&](const std::vector<InterpKey>& entry, const std::vector<int>& units, int count,
                          int chain) -> int {
          TRY(upload(e, d_entry, entry.data(), (size_t)npts));
          TRY(upload(e, d_units, units.data(), (size_t)count));
          const unsigned nb = chain ? 1u : (unsigned)((count + 63) / 64);
          if (x)
            KLAUNCH(NECGPU_K_PATTERN, 0.0,
                    near_field_chain_kernel<true><<<nb, chain ? 1 : 64, 0, e->stream>>>(
                        a, d_ax, e->d_somm, d_units, count, d_entry, e->d_interp_carry, d_rec, d_near, chain));
          else
            KLAUNCH(NECGPU_K_PATTERN, 0.0,
                    near_field_chain_kernel<false><<<nb, chain ? 1 : 64, 0, e->stream>>>(
                        a, d_ax, e->d_somm, d_units, count, d_entry, e->d_interp_carry, d_rec, d_near, chain));
          return 0;
        };
        if ((rc = resolve_cache_order(e, npts, d_rec, launch))) break;
        a.near = d_near;
      }
      switch (e->ground) {
        case kGroundNone: rc = x ? launch_near_e<kGroundNone, true>(e, a) : launch_near_e<kGroundNone, false>(e, a); break;
        case kGroundPerfect:
          rc = x ? launch_near_e<kGroundPerfect, true>(e, a) : launch_near_e<kGroundPerfect, false>(e, a);
          break;
        case kGroundReflection:
          rc = x ? launch_near_e<kGroundReflection, true>(e, a) : launch_near_e<kGroundReflection, false>(e, a);
          break;
        default:
          rc = x ? launch_near_e<kGroundSommerfeld, true>(e, a) : launch_near_e<kGroundSommerfeld, false>(e, a);
      }
      if (rc) break;
    }
    CUDA_TRY(cudaMemcpyAsync(fields, d_out, 3 * (size_t)npts * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
    int st = 0;
    if ((rc = sync_status(e, &st))) break;
    e->stats.d2h_bytes += 3 * (size_t)npts * sizeof(double2);
    if (st & kStatSommerfeldTab)
      rc = fail(e, NECGPU_ERR_UNSUPPORTED, "near_field: a point lies within 0.95 wavelength of a segment's ground "
                                           "image and no Sommerfeld tables are set");
    else if (st & kStatIterCap)
      rc = fail(e, NECGPU_ERR_NONFINITE, "near_field: quadrature did not terminate (non-finite point?)");
  } while (false);
  cleanup();
  return rc;
}

int necgpu_copy_sommerfeld(necgpu_engine* e, double* tables) {
  if (!e || !tables) return NECGPU_ERR_ARG;
  if (!e->somm_ready) return fail(e, NECGPU_ERR_ARG, "copy_sommerfeld: no tables");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemcpyAsync(tables, e->d_somm, kSommPoints * sizeof(cplx), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return NECGPU_OK;
}

int necgpu_reset_interpolation(necgpu_engine* e) {
  if (!e) return NECGPU_ERR_ARG;
  e->interp_key = InterpKey{kInterpFresh, 0, 0, 0};
  return NECGPU_OK;
}

int necgpu_copy_solution(necgpu_engine* e, double* x) {
  if (!e || !x) return NECGPU_ERR_ARG;
  if (!e->have_solution) return fail(e, NECGPU_ERR_ARG, "copy_solution: no solution held");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaMemcpyAsync(x, e->d_x, e->n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->stats.d2h_bytes += e->n * sizeof(double2);
  return NECGPU_OK;
}

int necgpu_adjoint_solve(necgpu_engine* e, int nrhs, const double* phi, double* w) {
  if (!e) return NECGPU_ERR_ARG;
  if (nrhs < 1 || !phi || !w) return fail(e, NECGPU_ERR_ARG, "adjoint: bad arguments");
  CUDA_TRY(cudaSetDevice(e->device));
  TRY(ensure_adjoint(e));
  const int64_t n = e->n;
  if (nrhs > e->adj_cap || !e->d_adj_r) {
    TRY(dalloc(e, e->d_adj_phi, (size_t)nrhs * n));
    TRY(dalloc(e, e->d_adj_w, (size_t)nrhs * n));
    TRY(dalloc(e, e->d_adj_r, (size_t)n));
    e->adj_cap = nrhs;
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_adj_phi, phi, (size_t)nrhs * n * sizeof(double2), cudaMemcpyHostToDevice, e->stream));
  e->stats.h2d_bytes += (int64_t)nrhs * n * sizeof(double2);
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  for (int k = 0; k < nrhs; k++) {
    int it = 0;
    double rel = 0.0;
    TRY(refine_T(e, e->d_adj_phi + (int64_t)k * n, e->d_adj_w + (int64_t)k * n, &it, &rel));
    e->stats.refine_iters = it;
    e->stats.refine_residual = rel;
    if (rel > 1e-6) return fail(e, NECGPU_ERR_REFINE, "adjoint: refinement did not converge");
  }
  CUDA_TRY(cudaMemcpyAsync(w, e->d_adj_w, (size_t)nrhs * n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += (int64_t)nrhs * n * sizeof(double2);
  int st = 0;
  TRY(sync_status(e, &st));
  if (st & (1 << 9)) return fail(e, NECGPU_ERR_CUDA, "adjoint: triangular sweep gave up waiting on a block");
  return NECGPU_OK;
}

int necgpu_pattern_weights(necgpu_engine* e, double theta, double phi, double* phi_t, double* phi_p) {
  if (!e) return NECGPU_ERR_ARG;
  if (!phi_t || !phi_p) return fail(e, NECGPU_ERR_ARG, "pattern_weights: null argument");
  if (e->n <= 0) return fail(e, NECGPU_ERR_ARG, "pattern_weights: no structure set");
  CUDA_TRY(cudaSetDevice(e->device));
  const int64_t n = e->n;
  if (!e->d_pwts) TRY(dalloc(e, e->d_pwts, 2 * (size_t)n));
  CUDA_TRY(cudaMemsetAsync(e->d_pwts, 0, 2 * n * sizeof(double2), e->stream));
  const FarDir d = engine_far_dir(e, theta, phi);
  double* pt = reinterpret_cast<double*>(e->d_pwts);
  KLAUNCH(NECGPU_K_PATTERN, (double)n * d.ksymp,
          pattern_weights_kernel<<<(unsigned)((n + 127) / 128), 128, 0, e->stream>>>(
              n, d, e->d_seg, e->d_cptr, e->d_cbasis, e->d_ccoef, e->d_ccoef + e->nc, e->d_ccoef + 2 * e->nc, pt,
              pt + 2 * n));
  CUDA_TRY(cudaMemcpyAsync(phi_t, e->d_pwts, n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaMemcpyAsync(phi_p, e->d_pwts + n, n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  e->stats.d2h_bytes += 2 * n * sizeof(double2);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  kflush(e);
  return NECGPU_OK;
}

int necgpu_perturbed_terms(necgpu_engine* e, int nstruct, const necgpu_structure* structs, int nw, const double* w,
                           double theta, double phi, double* zx, double* efar) {
  if (!e) return NECGPU_ERR_ARG;
  if (nstruct < 1 || nstruct > 65535 || !structs || nw < 0 || nw > kMaxContract || (nw > 0 && (!w || !zx)) || !efar)
    return fail(e, NECGPU_ERR_ARG, "perturbed_terms: bad arguments");
  if (!e->have_solution) return fail(e, NECGPU_ERR_ARG, "perturbed_terms: no solution held");
  CUDA_TRY(cudaSetDevice(e->device));
  const int64_t n = e->n, ne = e->ne, nc = e->nc;
  // every perturbed structure must share the held one's table layout and medium
  std::vector<double> seg((size_t)nstruct * 8 * n), pe((size_t)nstruct * 3 * std::max<int64_t>(ne, 1)),
      pc((size_t)nstruct * 3 * std::max<int64_t>(nc, 1));
  for (int q = 0; q < nstruct; q++) {
    const necgpu_structure* s = structs + q;
    if (s->n != n) return fail(e, NECGPU_ERR_ARG, "perturbed_terms: segment count differs from the held structure");
    if (s->ground != e->ground || (s->use_exk != 0) != (e->use_exk != 0) || s->rkh != e->P.rkh ||
        s->eta != e->P.eta || s->zrati_re != e->P.zrati.re || s->zrati_im != e->P.zrati.im ||
        s->frati_re != e->P.frati.re || s->frati_im != e->P.frati.im)
      return fail(e, NECGPU_ERR_ARG, "perturbed_terms: medium, ground or kernel settings differ from the held structure");
    if (!std::equal(s->trio_ptr, s->trio_ptr + n + 1, e->h_tptr.begin()) ||
        !std::equal(s->trio_basis, s->trio_basis + e->h_tptr[n], e->h_tbasis.begin()))
      return fail(e, NECGPU_ERR_ARG, "perturbed_terms: basis-table layout differs from the held structure");
    if (s->ek_ind1 && s->ek_ind2)
      for (int64_t i = 0; i < n; i++)
        if (s->ek_ind1[i] != e->h_ind[i] || s->ek_ind2[i] != e->h_ind[n + i])
          return fail(e, NECGPU_ERR_ARG, "perturbed_terms: extended-kernel end flags differ from the held structure");
    double* g = seg.data() + (size_t)q * 8 * n;
    const double* src[8] = {s->x, s->y, s->z, s->length, s->radius, s->cab, s->sab, s->salp};
    for (int a = 0; a < 8; a++) std::copy(src[a], src[a] + n, g + (size_t)a * n);
    TileLists TL;
    build_tile_lists(s, n, e->ntiles, TL);
    if ((int64_t)TL.ecol.size() != ne) return fail(e, NECGPU_ERR_ARG, "perturbed_terms: tile layout differs");
    std::copy(TL.ecoef.begin(), TL.ecoef.end(), pe.begin() + (size_t)q * 3 * std::max<int64_t>(ne, 1));
    CoefLists CL;
    build_coef_lists(s, n, CL);
    std::copy(CL.ccoef.begin(), CL.ccoef.end(), pc.begin() + (size_t)q * 3 * std::max<int64_t>(nc, 1));
  }
  const size_t pes = 3 * std::max<int64_t>(ne, 1), pcs = 3 * std::max<int64_t>(nc, 1);
  if (nstruct > e->p_cap) {
    TRY(dalloc(e, e->d_pseg, (size_t)nstruct * 8 * n));
    TRY(dalloc(e, e->d_pecoef, (size_t)nstruct * pes));
    TRY(dalloc(e, e->d_pccoef, (size_t)nstruct * pcs));
    TRY(dalloc(e, e->d_pout, (size_t)nstruct * 2 * kMaxContract));
    TRY(dalloc(e, e->d_pfar, (size_t)nstruct * 2));
    TRY(dalloc(e, e->d_pargs, (size_t)nstruct));
    TRY(dalloc(e, e->d_pcargs, (size_t)nstruct));
    e->p_cap = nstruct;
  }
  if (nw > e->pw_cap || !e->d_pw) {
    TRY(dalloc(e, e->d_pw, (size_t)std::max(nw, 1) * n));
    e->pw_cap = std::max(nw, 1);
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_pseg, seg.data(), seg.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_pecoef, pe.data(), pe.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_pccoef, pc.data(), pc.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream));
  if (nw > 0)
    CUDA_TRY(cudaMemcpyAsync(e->d_pw, w, (size_t)nw * n * sizeof(double2), cudaMemcpyHostToDevice, e->stream));
  e->stats.h2d_bytes += (int64_t)(seg.size() + pe.size() + pc.size()) * sizeof(double) + (int64_t)nw * n * 16;
  std::vector<FillArgs> fa(nstruct);
  std::vector<ContractArgs> ca(nstruct);
  for (int q = 0; q < nstruct; q++) {
    FillArgs& a = fa[q];
    const double* g = e->d_pseg + (size_t)q * 8 * n;
    a.n = n;
    a.ld = e->ld;
    a.x = g;
    a.y = g + n;
    a.z = g + 2 * n;
    a.s = g + 3 * n;
    a.b = g + 4 * n;
    a.cab = g + 5 * n;
    a.sab = g + 6 * n;
    a.salp = g + 7 * n;
    a.ind1 = e->d_ind;
    a.ind2 = e->d_ind + n;
    a.tile_src_ptr = e->d_tile_ptr;
    a.tsrc = e->d_tsrc;
    a.tsrc_eptr = e->d_tsrc_eptr;
    a.ecol = e->d_ecol;
    const double* c = e->d_pecoef + (size_t)q * pes;
    a.ea = c;
    a.eb = c + ne;
    a.ec = c + 2 * ne;
    a.P = e->P;
    a.P.near_g = nullptr;
    a.Z64 = nullptr;
    a.Z32 = nullptr;
    a.status = e->d_status;
    ca[q].x = e->d_x;
    ca[q].w = e->d_pw;
    ca[q].nw = nw;
    ca[q].out = e->d_pout + (size_t)q * 2 * kMaxContract;
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_pargs, fa.data(), fa.size() * sizeof(FillArgs), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_pcargs, ca.data(), ca.size() * sizeof(ContractArgs), cudaMemcpyHostToDevice,
                           e->stream));
  CUDA_TRY(cudaMemsetAsync(e->d_pout, 0, (size_t)nstruct * 2 * kMaxContract * sizeof(double), e->stream));
  CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
  if (nw > 0) {
    const dim3 grid((unsigned)((n + kFillTI - 1) / kFillTI), (unsigned)e->ntiles, (unsigned)nstruct);
    const bool xk = e->use_exk != 0;
#define NECB_CONTRACT(G)                                                                                      \
  (xk ? (fill_contract_kernel<G, true><<<grid, kFillTI, 0, e->stream>>>(e->d_pargs, e->d_pcargs), 0)           \
      : (fill_contract_kernel<G, false><<<grid, kFillTI, 0, e->stream>>>(e->d_pargs, e->d_pcargs), 0))
    switch (e->ground) {
      case kGroundNone: KLAUNCH(NECGPU_K_FILL, (double)nstruct * n * n, NECB_CONTRACT(kGroundNone)); break;
      case kGroundPerfect: KLAUNCH(NECGPU_K_FILL, (double)nstruct * n * n, NECB_CONTRACT(kGroundPerfect)); break;
      case kGroundReflection:
        KLAUNCH(NECGPU_K_FILL, (double)nstruct * n * n, NECB_CONTRACT(kGroundReflection));
        break;
      default: KLAUNCH(NECGPU_K_FILL, (double)nstruct * n * n, NECB_CONTRACT(kGroundSommerfeld)); break;
    }
#undef NECB_CONTRACT
  }
  const FarDir d = engine_far_dir(e, theta, phi);
  KLAUNCH(NECGPU_K_PATTERN, (double)nstruct * n * d.ksymp,
          far_batch_kernel<<<(unsigned)nstruct, kFarBatchThreads, 0, e->stream>>>(
              n, nc, d, e->d_pseg, e->d_cptr, e->d_cbasis, e->d_pccoef, e->d_x, e->d_pfar));
  if (nw > 0) {
    std::vector<double> out((size_t)nstruct * 2 * kMaxContract);
    CUDA_TRY(cudaMemcpyAsync(out.data(), e->d_pout, out.size() * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaMemcpyAsync(efar, e->d_pfar, (size_t)nstruct * 2 * sizeof(double2), cudaMemcpyDeviceToHost,
                             e->stream));
    int st = 0;
    TRY(sync_status(e, &st));
    for (int q = 0; q < nstruct; q++)
      for (int k = 0; k < nw; k++) {
        zx[((size_t)q * nw + k) * 2] = out[(size_t)q * 2 * kMaxContract + 2 * k];
        zx[((size_t)q * nw + k) * 2 + 1] = out[(size_t)q * 2 * kMaxContract + 2 * k + 1];
      }
    if (st & kStatSommerfeldTab)
      return fail(e, NECGPU_ERR_UNSUPPORTED, "perturbed_terms: a segment pair needs the Sommerfeld table path");
    if (st & kStatIterCap) return fail(e, NECGPU_ERR_NONFINITE, "perturbed_terms: quadrature did not terminate");
  } else {
    CUDA_TRY(cudaMemcpyAsync(efar, e->d_pfar, (size_t)nstruct * 2 * sizeof(double2), cudaMemcpyDeviceToHost,
                             e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
  }
  e->stats.d2h_bytes += (int64_t)nstruct * (2 * kMaxContract * 8 + 32);
  kflush(e);
  return NECGPU_OK;
}

int necgpu_batch_solve(necgpu_engine* e, int nprob, const necgpu_structure* structs, const double* rhs,
                       const int* feed, const double* volt, const double* wavelength, int ndir, const double* theta,
                       const double* phi, double* cur, float* gain, double* eth, double* eph, int* status,
                       double* residual) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (nprob < 1 || nprob > 65535 || !structs || !rhs || !cur || !status || ndir < 0 ||
      (ndir > 0 && (!theta || !phi || (!eth) != (!eph))) || (gain && (!feed || !volt || !wavelength)))
    return fail(e, NECGPU_ERR_ARG, "batch_solve: bad arguments");
  CUDA_TRY(cudaSetDevice(e->device));
  const necgpu_structure& s0 = structs[0];
  // host tables of every problem, concatenated
  std::vector<int64_t> seg_off(nprob + 1, 0), z_off(nprob + 1, 0);
  for (int p = 0; p < nprob; p++) {
    const necgpu_structure& s = structs[p];
    if (s.n < 2 || s.n > kBatchMaxN)
      return fail(e, NECGPU_ERR_ARG, "batch_solve: problem " + std::to_string(p) + " has " + std::to_string(s.n) +
                                         " segments; the batched path takes 2.." + std::to_string(kBatchMaxN));
    if (s.ground != s0.ground || (s.use_exk != 0) != (s0.use_exk != 0) || s.eta != s0.eta ||
        s.zrati_re != s0.zrati_re || s.zrati_im != s0.zrati_im)
      return fail(e, NECGPU_ERR_ARG, "batch_solve: all problems must share the medium, ground and kernel settings");
    seg_off[p + 1] = seg_off[p] + s.n;
    z_off[p + 1] = z_off[p] + s.n * s.n;
  }
  const int64_t T = seg_off[nprob], Zt = z_off[nprob];
  std::vector<double> seg(8 * T);
  std::vector<int32_t> ind(2 * T, 0);
  std::vector<int32_t> tp_pool, ts_pool, te_pool, cptr_g(T + 1, 0), cbasis_pool;
  std::vector<uint8_t> ecol_pool;
  std::vector<double> ecoef_pool, ca_pool, cb_pool, cc_pool;
  std::vector<int64_t> tp_off(nprob), ts_off(nprob), te_off(nprob), ec_off(nprob), ecf_off(nprob), ne_p(nprob);
  std::vector<int> ntiles_p(nprob), seg_prob(T);
  // per-problem tile and coefficient lists on all host cores, then concatenated
  std::vector<TileLists> TLs(nprob);
  std::vector<CoefLists> CLs(nprob);
  std::vector<int> bad(nprob, 0);
  {
    const int nth = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 64));
    std::atomic<int> nextp(0);
    auto work = [&]() {
      for (int p = nextp++; p < nprob; p = nextp++) {
        const necgpu_structure& s = structs[p];
        const int64_t n = s.n;
        const int32_t* tp = s.trio_ptr;
        bool ok = tp[0] == 0;
        for (int64_t j = 0; ok && j < n; j++) ok = tp[j + 1] >= tp[j];
        for (int64_t k = 0; ok && k < tp[n]; k++) ok = s.trio_basis[k] >= 0 && s.trio_basis[k] < n;
        if (!ok) {
          bad[p] = 1;
          continue;
        }
        build_tile_lists(&s, n, (int)((n + kFillTB - 1) / kFillTB), TLs[p]);
        build_coef_lists(&s, n, CLs[p]);
      }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < nth; i++) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
  }
  for (int p = 0; p < nprob; p++)
    if (bad[p]) return fail(e, NECGPU_ERR_ARG, "batch_solve: basis tables of problem " + std::to_string(p) + " are malformed");
  for (int p = 0; p < nprob; p++) {
    const necgpu_structure& s = structs[p];
    const int64_t n = s.n, o = seg_off[p];
    const double* src[8] = {s.x, s.y, s.z, s.length, s.radius, s.cab, s.sab, s.salp};
    for (int a = 0; a < 8; a++) std::copy(src[a], src[a] + n, seg.begin() + a * T + o);
    if (s.ek_ind1 && s.ek_ind2) {
      std::copy(s.ek_ind1, s.ek_ind1 + n, ind.begin() + o);
      std::copy(s.ek_ind2, s.ek_ind2 + n, ind.begin() + T + o);
    }
    for (int64_t j = 0; j < n; j++) seg_prob[o + j] = p;
    const int32_t* tp = s.trio_ptr;
    ntiles_p[p] = (int)((n + kFillTB - 1) / kFillTB);
    const TileLists& TL = TLs[p];
    tp_off[p] = (int64_t)tp_pool.size();
    ts_off[p] = (int64_t)ts_pool.size();
    te_off[p] = (int64_t)te_pool.size();
    ec_off[p] = (int64_t)ecol_pool.size();
    ecf_off[p] = (int64_t)ecoef_pool.size();
    ne_p[p] = (int64_t)TL.ecol.size();
    tp_pool.insert(tp_pool.end(), TL.tile_ptr.begin(), TL.tile_ptr.end());
    ts_pool.insert(ts_pool.end(), TL.tsrc.begin(), TL.tsrc.end());
    te_pool.insert(te_pool.end(), TL.tsrc_eptr.begin(), TL.tsrc_eptr.end());
    ecol_pool.insert(ecol_pool.end(), TL.ecol.begin(), TL.ecol.end());
    ecoef_pool.insert(ecoef_pool.end(), TL.ecoef.begin(), TL.ecoef.end());
    const CoefLists& CL = CLs[p];
    const int64_t nt = tp[n], cbase = (int64_t)cbasis_pool.size();
    for (int64_t j = 0; j < n; j++) cptr_g[o + j] = (int32_t)(cbase + CL.cptr[j]);
    cbasis_pool.insert(cbasis_pool.end(), CL.cbasis.begin(), CL.cbasis.begin() + nt);
    ca_pool.insert(ca_pool.end(), CL.ccoef.begin(), CL.ccoef.begin() + nt);
    cb_pool.insert(cb_pool.end(), CL.ccoef.begin() + nt, CL.ccoef.begin() + 2 * nt);
    cc_pool.insert(cc_pool.end(), CL.ccoef.begin() + 2 * nt, CL.ccoef.begin() + 3 * nt);
  }
  cptr_g[T] = (int32_t)cbasis_pool.size();
  for (auto* v : {&ts_pool, &te_pool, &cbasis_pool})
    if (v->empty()) v->push_back(0);
  if (ecol_pool.empty()) ecol_pool.push_back(0);
  for (auto* v : {&ca_pool, &cb_pool, &cc_pool, &ecoef_pool})
    if (v->empty()) v->push_back(0.0);
  // device pools (stream-ordered; freed at the end of the call)
  double *d_seg = nullptr, *d_ecoef = nullptr, *d_ca = nullptr, *d_cb = nullptr, *d_cc = nullptr, *d_abc = nullptr,
         *d_res = nullptr;
  int32_t *d_ind = nullptr, *d_tp = nullptr, *d_ts = nullptr, *d_te = nullptr, *d_cptr = nullptr, *d_cbasis = nullptr;
  uint8_t* d_ecol = nullptr;
  double2 *d_Z64 = nullptr, *d_b = nullptr, *d_x = nullptr, *d_cur = nullptr, *d_eth = nullptr, *d_eph = nullptr,
          *d_dirs = nullptr;
  float2* d_Z32 = nullptr;
  int *d_perm = nullptr, *d_segp = nullptr, *d_order = nullptr, *d_next = nullptr, *d_st = nullptr;
  BatchProblem* d_probs = nullptr;
  FillArgs* d_args = nullptr;
  int4* d_items = nullptr;
  auto release = [&]() {
    dfree(e, d_seg), dfree(e, d_ecoef), dfree(e, d_ca), dfree(e, d_cb), dfree(e, d_cc), dfree(e, d_abc);
    dfree(e, d_res), dfree(e, d_ind), dfree(e, d_tp), dfree(e, d_ts), dfree(e, d_te), dfree(e, d_cptr);
    dfree(e, d_cbasis), dfree(e, d_ecol), dfree(e, d_Z64), dfree(e, d_b), dfree(e, d_x), dfree(e, d_cur);
    dfree(e, d_eth), dfree(e, d_eph), dfree(e, d_dirs), dfree(e, d_Z32), dfree(e, d_perm), dfree(e, d_segp);
    dfree(e, d_order), dfree(e, d_next), dfree(e, d_st), dfree(e, d_probs), dfree(e, d_args), dfree(e, d_items);
  };
  int rc = 0;
  do {
    if ((rc = upload(e, d_seg, seg.data(), seg.size()))) break;
    if ((rc = upload(e, d_ind, ind.data(), ind.size()))) break;
    if ((rc = upload(e, d_tp, tp_pool.data(), tp_pool.size()))) break;
    if ((rc = upload(e, d_ts, ts_pool.data(), ts_pool.size()))) break;
    if ((rc = upload(e, d_te, te_pool.data(), te_pool.size()))) break;
    if ((rc = upload(e, d_ecol, ecol_pool.data(), ecol_pool.size()))) break;
    if ((rc = upload(e, d_ecoef, ecoef_pool.data(), ecoef_pool.size()))) break;
    if ((rc = upload(e, d_cptr, cptr_g.data(), cptr_g.size()))) break;
    if ((rc = upload(e, d_cbasis, cbasis_pool.data(), cbasis_pool.size()))) break;
    if ((rc = upload(e, d_ca, ca_pool.data(), ca_pool.size()))) break;
    if ((rc = upload(e, d_cb, cb_pool.data(), cb_pool.size()))) break;
    if ((rc = upload(e, d_cc, cc_pool.data(), cc_pool.size()))) break;
    if ((rc = upload(e, d_segp, seg_prob.data(), seg_prob.size()))) break;
    if ((rc = upload(e, d_b, reinterpret_cast<const double2*>(rhs), (size_t)T))) break;
    if ((rc = dalloc(e, d_Z64, (size_t)Zt))) break;
    if ((rc = dalloc(e, d_Z32, (size_t)Zt))) break;
    if ((rc = dalloc(e, d_x, (size_t)T))) break;
    if ((rc = dalloc(e, d_perm, (size_t)T))) break;
    if ((rc = dalloc(e, d_cur, (size_t)T))) break;
    if ((rc = dalloc(e, d_abc, 6 * (size_t)T))) break;
    if ((rc = dalloc(e, d_st, (size_t)nprob))) break;
    if ((rc = dalloc(e, d_res, (size_t)nprob))) break;
    if ((rc = dalloc(e, d_next, 1))) break;
    // per-problem fill arguments and the fill work list
    std::vector<FillArgs> fa(nprob);
    std::vector<BatchProblem> bp(nprob);
    std::vector<int4> items;
    for (int p = 0; p < nprob; p++) {
      const necgpu_structure& s = structs[p];
      const int64_t n = s.n, o = seg_off[p];
      FillArgs& a = fa[p];
      a.n = n;
      a.ld = n;
      a.x = d_seg + o;
      a.y = d_seg + T + o;
      a.z = d_seg + 2 * T + o;
      a.s = d_seg + 3 * T + o;
      a.b = d_seg + 4 * T + o;
      a.cab = d_seg + 5 * T + o;
      a.sab = d_seg + 6 * T + o;
      a.salp = d_seg + 7 * T + o;
      a.ind1 = d_ind + o;
      a.ind2 = d_ind + T + o;
      a.tile_src_ptr = d_tp + tp_off[p];
      a.tsrc = d_ts + ts_off[p];
      a.tsrc_eptr = d_te + te_off[p];
      a.ecol = d_ecol + ec_off[p];
      a.ea = d_ecoef + ecf_off[p];
      a.eb = a.ea + ne_p[p];
      a.ec = a.ea + 2 * ne_p[p];
      a.P.rkh = s.rkh;
      a.P.eta = s.eta;
      a.P.zrati = mk(s.zrati_re, s.zrati_im);
      a.P.frati = mk(s.frati_re, s.frati_im);
      a.P.u = a.P.zrati;
      a.P.u2 = a.P.zrati * a.P.zrati;
      a.Z64 = d_Z64 + z_off[p];
      a.Z32 = d_Z32 + z_off[p];
      a.status = e->d_status;
      bp[p] = BatchProblem{(int)n, z_off[p], o};
      const int rt = (int)((n + kFillTI - 1) / kFillTI);
      for (int r = 0; r < rt; r++)
        for (int c = 0; c < ntiles_p[p]; c++) items.push_back(make_int4(p, r, c, 0));
    }
    std::vector<int> order(nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return structs[a].n > structs[b].n; });
    if ((rc = upload(e, d_args, fa.data(), fa.size()))) break;
    if ((rc = upload(e, d_probs, bp.data(), bp.size()))) break;
    if ((rc = upload(e, d_items, items.data(), items.size()))) break;
    if ((rc = upload(e, d_order, order.data(), order.size()))) break;
    CUDA_TRY(cudaMemsetAsync(e->d_status, 0, 4 * sizeof(int), e->stream));
    CUDA_TRY(cudaMemsetAsync(d_next, 0, sizeof(int), e->stream));
    // fill
    const bool xk = s0.use_exk != 0;
    const double pairs = (double)0 + [&] {
      double q = 0;
      for (int p = 0; p < nprob; p++) q += (double)structs[p].n * structs[p].n;
      return q;
    }();
#define NECB_BFILL(G)                                                                                         \
  (xk ? (batch_fill_kernel<G, true><<<(unsigned)items.size(), kFillTI, 0, e->stream>>>(d_args, d_items), 0)    \
      : (batch_fill_kernel<G, false><<<(unsigned)items.size(), kFillTI, 0, e->stream>>>(d_args, d_items), 0))
    switch (s0.ground) {
      case kGroundNone: KLAUNCH(NECGPU_K_FILL, pairs, NECB_BFILL(kGroundNone)); break;
      case kGroundPerfect: KLAUNCH(NECGPU_K_FILL, pairs, NECB_BFILL(kGroundPerfect)); break;
      case kGroundReflection: KLAUNCH(NECGPU_K_FILL, pairs, NECB_BFILL(kGroundReflection)); break;
      default: KLAUNCH(NECGPU_K_FILL, pairs, NECB_BFILL(kGroundSommerfeld)); break;
    }
#undef NECB_BFILL
    // LU and refined solve, one problem per CTA at a time
    CUDA_TRY(cudaFuncSetAttribute(batch_lu_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kBatchSmem));
    double lu_flops = 0;
    for (int p = 0; p < nprob; p++) lu_flops += 8.0 * std::pow((double)structs[p].n, 3) / 3.0;
    KLAUNCH(NECGPU_K_PANEL, lu_flops,
            batch_lu_solve_kernel<<<(unsigned)std::min(nprob, e->nsm), kBatchThreads, kBatchSmem, e->stream>>>(
                nprob, d_order, d_probs, d_Z32, d_Z64, d_perm, d_b, d_x, e->refine_tol, d_next, d_st, d_res));
    KLAUNCH(NECGPU_K_OTHER, 0.0,
            batch_coeff_kernel<<<(unsigned)((T + 255) / 256), 256, 0, e->stream>>>(
                T, d_segp, d_probs, d_cptr, d_cbasis, d_ca, d_cb, d_cc, d_x, d_abc, d_cur));
    double* d_gcop = nullptr;
    float* d_gain = nullptr;
    int64_t* d_so = nullptr;
    if (ndir > 0 && gain) {
      std::vector<int> fd(feed, feed + nprob);
      for (int p = 0; p < nprob; p++)
        if (fd[p] < 0 || fd[p] >= structs[p].n) {
          rc = fail(e, NECGPU_ERR_ARG, "batch_solve: feed segment out of range");
          break;
        }
      if (rc) break;
      int* d_feed = nullptr;
      double2* d_volt = nullptr;
      double* d_lam = nullptr;
      if ((rc = upload(e, d_feed, fd.data(), fd.size()))) break;
      if ((rc = upload(e, d_volt, reinterpret_cast<const double2*>(volt), (size_t)nprob))) break;
      if ((rc = upload(e, d_lam, wavelength, (size_t)nprob))) break;
      if ((rc = upload(e, d_so, seg_off.data(), seg_off.size()))) break;
      if ((rc = dalloc(e, d_gcop, (size_t)nprob))) break;
      KLAUNCH(NECGPU_K_OTHER, 0.0,
              batch_gain_norm_kernel<<<(unsigned)((nprob + 127) / 128), 128, 0, e->stream>>>(
                  nprob, d_so, d_feed, d_volt, d_lam, s0.eta, d_cur, d_gcop));
      dfree(e, d_feed);
      dfree(e, d_volt);
      dfree(e, d_lam);
      if ((rc = dalloc(e, d_gain, (size_t)nprob * ndir))) break;
    }
    if (ndir > 0) {
      std::vector<double> dirs(2 * (size_t)ndir);
      std::copy(theta, theta + ndir, dirs.begin());
      std::copy(phi, phi + ndir, dirs.begin() + ndir);
      double* dd = nullptr;
      if ((rc = upload(e, dd, dirs.data(), dirs.size()))) break;
      d_dirs = reinterpret_cast<double2*>(dd);
      if (eth) {
        if ((rc = dalloc(e, d_eth, (size_t)nprob * ndir))) break;
        if ((rc = dalloc(e, d_eph, (size_t)nprob * ndir))) break;
      }
      BatchPatternArgs pa{};
      pa.nprob = nprob;
      pa.ndir = ndir;
      pa.theta = dd;
      pa.phi = dd + ndir;
      if (!d_so && (rc = upload(e, d_so, seg_off.data(), seg_off.size()))) break;
      pa.seg_off = d_so;
      pa.seg = d_seg;
      pa.abc = d_abc;
      pa.nseg_total = T;
      pa.ksymp = s0.ground == kGroundNone ? 1 : 2;
      pa.perfect = s0.ground == kGroundPerfect ? 1 : 0;
      pa.zrati = mk(s0.zrati_re, s0.zrati_im);
      pa.eta = s0.eta;
      pa.eth = d_eth;
      pa.eph = d_eph;
      pa.gcop = d_gcop;
      pa.gain = d_gain;
      const dim3 g((unsigned)((ndir + kPatDirs - 1) / kPatDirs), (unsigned)nprob);
      KLAUNCH(NECGPU_K_PATTERN, (double)ndir * T * pa.ksymp,
              batch_pattern_kernel<<<g, kPatDirs * 32, 0, e->stream>>>(pa));
      if (eth) {
        CUDA_TRY(cudaMemcpyAsync(eth, d_eth, (size_t)nprob * ndir * sizeof(double2), cudaMemcpyDeviceToHost,
                                 e->stream));
        CUDA_TRY(cudaMemcpyAsync(eph, d_eph, (size_t)nprob * ndir * sizeof(double2), cudaMemcpyDeviceToHost,
                                 e->stream));
      }
      if (gain)
        CUDA_TRY(cudaMemcpyAsync(gain, d_gain, (size_t)nprob * ndir * sizeof(float), cudaMemcpyDeviceToHost,
                                 e->stream));
    }
    CUDA_TRY(cudaMemcpyAsync(cur, d_cur, (size_t)T * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaMemcpyAsync(status, d_st, (size_t)nprob * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    if (residual)
      CUDA_TRY(cudaMemcpyAsync(residual, d_res, (size_t)nprob * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    int st = 0;
    rc = sync_status(e, &st);
    dfree(e, d_gcop);
    dfree(e, d_gain);
    dfree(e, d_so);
    if (rc) break;
    kflush(e);
    if (st & kStatSommerfeldTab)
      rc = fail(e, NECGPU_ERR_UNSUPPORTED, "batch_solve: a segment pair needs the Sommerfeld table path");
    else if (st & kStatIterCap)
      rc = fail(e, NECGPU_ERR_NONFINITE, "batch_solve: quadrature did not terminate");
  } while (false);
  release();
  if (rc == 0) CUDA_TRY(cudaStreamSynchronize(e->stream));
  return rc;
}

int necgpu_read_resident(necgpu_engine* e, double* cur, double* eth, double* eph) {
  if (!e) return NECGPU_ERR_ARG;
  CUDA_TRY(cudaSetDevice(e->device));
  if (cur) CUDA_TRY(cudaMemcpyAsync(cur, e->d_cur, e->n * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  if (eth && e->res_ndir > 0)
    CUDA_TRY(cudaMemcpyAsync(eth, e->d_eth, e->res_ndir * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  if (eph && e->res_ndir > 0)
    CUDA_TRY(cudaMemcpyAsync(eph, e->d_eph, e->res_ndir * sizeof(double2), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return NECGPU_OK;
}

}  // extern "C"

// ---------------- allocation-free solve ----------------
// necgpu_solve_noalloc: the solve of necgpu_solve on the held factors, with
// the right-hand side and the results in caller-owned device memory and every
// scratch vector in one static device array, so that no call after the first
// allocates host or device memory.
namespace {

// Largest system the static scratch holds, and its layout (byte offsets):
// x and r (complex128), two complex64 work vectors, the 6n coefficient
// doubles used when the caller passes none, the residual norms and status
// words, and one flag word per 64-row block of the triangular sweeps.
constexpr int64_t kNoAllocMaxN = 16384;
static_assert(kNoAllocMaxN % kTrsvB == 0, "flag words per sweep block");
constexpr size_t kNoAllocOffX = 0;
constexpr size_t kNoAllocOffR = kNoAllocOffX + 16 * kNoAllocMaxN;
constexpr size_t kNoAllocOffW1 = kNoAllocOffR + 16 * kNoAllocMaxN;
constexpr size_t kNoAllocOffW2 = kNoAllocOffW1 + 8 * kNoAllocMaxN;
constexpr size_t kNoAllocOffAbc = kNoAllocOffW2 + 8 * kNoAllocMaxN;
constexpr size_t kNoAllocOffMisc = kNoAllocOffAbc + 48 * kNoAllocMaxN;  // rn2: 2 doubles, status: 4 ints
constexpr size_t kNoAllocOffFlags = kNoAllocOffMisc + 256;
constexpr size_t kNoAllocFlagBytes = sizeof(int) * (kNoAllocMaxN / kTrsvB);
constexpr size_t kNoAllocBytes = kNoAllocOffFlags + kNoAllocFlagBytes;  // 1,574,144 bytes

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch on this device
  int sweep_per_sm[2] = {0, 0};   // resident sweep CTAs per SM: [0] complex64, [1] complex128
  int epoch = 0;                  // last flag epoch of the sweeps on this device
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mutex;

// Every kernel the allocation-free solve can launch, FP64 and mixed.  With
// CUDA's lazy module loading (the default since CUDA 12.2) a kernel's code is
// loaded, and device memory taken for it, on its first launch; querying its
// attributes loads it, so the set-up touches each of them once.
int noalloc_preload(necgpu_engine* e) {
  const void* kernels[] = {
      (const void*)trsv_sweep_kernel<float2, true>,  (const void*)trsv_sweep_kernel<float2, false>,
      (const void*)trsv_sweep_kernel<double2, true>, (const void*)trsv_sweep_kernel<double2, false>,
      (const void*)permute_kernel<double2, double2>, (const void*)permute_kernel<float2, double2>,
      (const void*)norm2_kernel,                     (const void*)axpy_kernel<float2>,
      (const void*)residual_kernel,                  (const void*)coeff_kernel};
  for (const void* k : kernels) {
    cudaFuncAttributes fa;
    CUDA_TRY(cudaFuncGetAttributes(&fa, k));
  }
  return 0;
}

// The driver's cuMemGetAddressRange (base and size of the allocation that
// holds a device address), looked up once through the runtime.
typedef CUresult (*AddressRangeFn)(CUdeviceptr*, size_t*, CUdeviceptr);
AddressRangeFn address_range() {
  static AddressRangeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (AddressRangeFn)p;
  }
  return fn;
}

// Once per device, with that device current: look up the scratch array,
// zero its flag words (a sweep waits for a flag equal to its epoch, and the
// first epoch is 1), load every kernel of the path, set the sweep kernels'
// shared-memory limits and size their cooperative grids.
int noalloc_setup(necgpu_engine* e, NoAllocDevice** out) {
  if (e->device < 0 || e->device >= kNoAllocMaxDevices)
    return fail(e, NECGPU_ERR_ARG, "solve_noalloc: device index beyond the per-device table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocDevice& d = g_noalloc_dev[e->device];
  if (!d.base) {
    void* p = nullptr;
    CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (reinterpret_cast<uintptr_t>(p) & 255)
      return fail(e, NECGPU_ERR_CUDA, "solve_noalloc: static scratch is not 256-byte aligned");
    constexpr size_t dsm32 = trsv_diag_smem<float2>(), dsm64 = trsv_diag_smem<double2>();
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<float2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dsm32));
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<float2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dsm32));
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<double2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dsm64));
    CUDA_TRY(cudaFuncSetAttribute(trsv_sweep_kernel<double2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dsm64));
    int per_sm[2] = {0, 0};
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], trsv_sweep_kernel<float2, true>,
                                                           kSweepThreads, dsm32));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], trsv_sweep_kernel<double2, true>,
                                                           kSweepThreads, dsm64));
    if (per_sm[0] < 1 || per_sm[1] < 1) return fail(e, NECGPU_ERR_CUDA, "solve_noalloc: sweep kernel cannot be resident");
    TRY(noalloc_preload(e));
    if (!address_range()) return fail(e, NECGPU_ERR_CUDA, "solve_noalloc: cuMemGetAddressRange unavailable");
    unsigned char* base = static_cast<unsigned char*>(p);
    CUDA_TRY(cudaMemsetAsync(base + kNoAllocOffFlags, 0, kNoAllocFlagBytes, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    d.sweep_per_sm[0] = per_sm[0];
    d.sweep_per_sm[1] = per_sm[1];
    d.epoch = 0;
    d.base = base;
  }
  *out = &d;
  return 0;
}

// Forward and backward sweeps over the held factors M (the kernels of the
// engine's own solves) with the flag words in the static scratch.  rhs is
// consumed; the solution lands in sol.
template <typename T>
int noalloc_sweeps(necgpu_engine* e, NoAllocDevice& d, const T* M, T* rhs, T* sol, int* flags, int* status) {
  const int64_t n = e->n, ld = e->ld;
  const int nblk = (int)((n + kTrsvB - 1) / kTrsvB);
  constexpr bool f64 = std::is_same<T, double2>::value;
  constexpr size_t dsm = trsv_diag_smem<T>();
  const int grid = std::max(1, std::min(nblk, d.sweep_per_sm[f64 ? 1 : 0] * e->nsm));
  if (d.epoch > (1 << 30)) {  // restart the epochs long before the counter wraps
    CUDA_TRY(cudaMemsetAsync(flags, 0, kNoAllocFlagBytes, e->stream));
    d.epoch = 0;
  }
  for (int pass = 0; pass < 2; pass++) {
    int epoch;
    {
      std::lock_guard<std::mutex> lock(g_noalloc_mutex);  // the epoch counter is shared by the device's engines
      epoch = ++d.epoch;
    }
    const T* src = pass == 0 ? rhs : sol;
    T* dst = pass == 0 ? sol : rhs;
    void* args[] = {(void*)&M, (void*)&ld, (void*)&n, (void*)&src, (void*)&dst, (void*)&flags, (void*)&epoch,
                    (void*)&status};
    CUDA_TRY(cudaLaunchCooperativeKernel(pass == 0 ? (const void*)trsv_sweep_kernel<T, true>
                                                   : (const void*)trsv_sweep_kernel<T, false>,
                                         dim3(grid), dim3(kSweepThreads), args, dsm, e->stream));
    LAUNCHED();
  }
  CUDA_TRY(cudaMemcpyAsync(sol, rhs, n * sizeof(T), cudaMemcpyDeviceToDevice, e->stream));
  return 0;
}

int noalloc_device_buffer(necgpu_engine* e, const void* p, size_t bytes, size_t align, const char* what) {
  if (reinterpret_cast<uintptr_t>(p) % align)
    return fail(e, NECGPU_ERR_ARG, std::string("solve_noalloc: ") + what + " is not aligned");
  cudaPointerAttributes at;
  CUDA_TRY(cudaPointerGetAttributes(&at, p));
  if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != e->device)
    return fail(e, NECGPU_ERR_ARG, std::string("solve_noalloc: ") + what + " is not device memory of the engine's device");
  // the buffer must end inside the allocation that holds its start (a
  // caching allocator's sub-allocation is checked against its segment only)
  CUdeviceptr base = 0;
  size_t size = 0;
  if (address_range()(&base, &size, (CUdeviceptr)p) != CUDA_SUCCESS)
    return fail(e, NECGPU_ERR_ARG, std::string("solve_noalloc: ") + what + " is not inside a device allocation");
  if ((CUdeviceptr)p - base + bytes > size)
    return fail(e, NECGPU_ERR_ARG, std::string("solve_noalloc: ") + what + " ends beyond its allocation (needs " +
                                       std::to_string(bytes) + " bytes)");
  return 0;
}

bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a), b0 = reinterpret_cast<uintptr_t>(b);
  return a0 < b0 + nb && b0 < a0 + na;
}

}  // namespace

extern "C" {

int necgpu_solve_noalloc(necgpu_engine* e, const double* rhs_dev, double* cur_dev, double* abc_dev) {
  if (!e) return NECGPU_ERR_ARG;
  e->touched = true;  // a setting or use that a pooled engine must not carry over
  if (!rhs_dev || !cur_dev) return fail(e, NECGPU_ERR_ARG, "solve_noalloc: null argument");
  const int64_t n = e->n;
  if (n > kNoAllocMaxN)
    return fail(e, NECGPU_ERR_ARG,
                "solve_noalloc: n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                    std::to_string(kNoAllocMaxN) + " unknowns; use necgpu_solve");
  if (e->factored != NECGPU_FP64 && e->factored != NECGPU_MIXED)
    return fail(e, NECGPU_ERR_ARG, "solve_noalloc: no factorisation held");
  CUDA_TRY(cudaSetDevice(e->device));
  NoAllocDevice* d = nullptr;
  TRY(noalloc_setup(e, &d));
  const size_t vec = (size_t)n * sizeof(double2);
  TRY(noalloc_device_buffer(e, rhs_dev, vec, 16, "rhs"));
  TRY(noalloc_device_buffer(e, cur_dev, vec, 16, "cur"));
  if (abc_dev) TRY(noalloc_device_buffer(e, abc_dev, 6 * (size_t)n * sizeof(double), 8, "abc"));
  if (overlaps(rhs_dev, vec, cur_dev, vec) || (abc_dev && (overlaps(abc_dev, 48 * (size_t)n, rhs_dev, vec) ||
                                                           overlaps(abc_dev, 48 * (size_t)n, cur_dev, vec))))
    return fail(e, NECGPU_ERR_ARG, "solve_noalloc: rhs, cur and abc must not overlap");
  unsigned char* base = d->base;
  double2* x = reinterpret_cast<double2*>(base + kNoAllocOffX);
  double2* r = reinterpret_cast<double2*>(base + kNoAllocOffR);
  float2* w1 = reinterpret_cast<float2*>(base + kNoAllocOffW1);
  float2* w2 = reinterpret_cast<float2*>(base + kNoAllocOffW2);
  double* abc = abc_dev ? abc_dev : reinterpret_cast<double*>(base + kNoAllocOffAbc);
  double* rn2 = reinterpret_cast<double*>(base + kNoAllocOffMisc);
  int* status = reinterpret_cast<int*>(base + kNoAllocOffMisc + 2 * sizeof(double));
  int* flags = reinterpret_cast<int*>(base + kNoAllocOffFlags);
  const double2* b = reinterpret_cast<const double2*>(rhs_dev);
  const unsigned g1 = (unsigned)((n + 255) / 256);
  CUDA_TRY(cudaMemsetAsync(status, 0, 4 * sizeof(int), e->stream));
  int iters = 0;
  double rel = 0.0;
  if (e->factored == NECGPU_FP64) {
    permute_kernel<double2, double2><<<g1, 256, 0, e->stream>>>(b, e->d_perm, r, n);
    LAUNCHED();
    TRY(noalloc_sweeps<double2>(e, *d, e->Z64, r, x, flags, status));
  } else {
    // the refinement of the engine's mixed solve, on the static vectors
    CUDA_TRY(cudaMemsetAsync(x, 0, vec, e->stream));
    CUDA_TRY(cudaMemcpyAsync(r, b, vec, cudaMemcpyDeviceToDevice, e->stream));
    CUDA_TRY(cudaMemsetAsync(rn2, 0, 2 * sizeof(double), e->stream));
    norm2_kernel<<<g1, 256, 0, e->stream>>>(b, n, rn2 + 1);
    LAUNCHED();
    const unsigned gr = (unsigned)std::min<int64_t>((n + 7) / 8, 8 * e->nsm);
    double prev = 1e300;
    rel = 1.0;
    for (; iters <= e->refine_max; iters++) {
      permute_kernel<float2, double2><<<g1, 256, 0, e->stream>>>(r, e->d_perm, w1, n);
      LAUNCHED();
      TRY(noalloc_sweeps<float2>(e, *d, e->Z32, w1, w2, flags, status));
      axpy_kernel<float2><<<g1, 256, 0, e->stream>>>(x, w2, n);
      LAUNCHED();
      CUDA_TRY(cudaMemsetAsync(rn2, 0, sizeof(double), e->stream));
      residual_kernel<<<gr, 256, 0, e->stream>>>(e->Z64, e->ld, n, x, b, r, rn2);
      LAUNCHED();
      struct {
        double rn2[2];
        int status[4];
      } h{};  // the norms and the status words are adjacent in the scratch
      static_assert(sizeof(h) == 2 * sizeof(double) + 4 * sizeof(int), "misc block layout");
      CUDA_TRY(cudaMemcpyAsync(&h, rn2, sizeof(h), cudaMemcpyDeviceToHost, e->stream));
      CUDA_TRY(cudaStreamSynchronize(e->stream));
      if (h.status[0]) return fail(e, NECGPU_ERR_CUDA, "solve_noalloc: triangular sweep gave up waiting on a block");
      const double bn = std::sqrt(h.rn2[1]);
      rel = bn > 0 ? std::sqrt(h.rn2[0]) / bn : 0.0;
      if (!std::isfinite(rel)) return fail(e, NECGPU_ERR_NONFINITE, "solve_noalloc: non-finite residual");
      if (rel <= e->refine_tol || rel > 0.5 * prev) {
        iters++;
        break;
      }
      prev = rel;
    }
    if (e->tc_format_used == 2 && iters > e->tf32_max_iters) e->tf32_demoted = true;
    if (e->blockpiv && rel > kRefineFallback)
      return fail(e, NECGPU_ERR_REFINE,
                  "solve_noalloc: refinement stalled on the block-pivoted factors; necgpu_solve refactors "
                  "with partial pivoting, after which this call converges");
    if (rel > 1e-6) return fail(e, NECGPU_ERR_REFINE, "solve_noalloc: refinement did not converge");
  }
  coeff_kernel<<<g1, 256, 0, e->stream>>>(n, e->d_cptr, e->d_cbasis, e->d_ccoef, e->d_ccoef + e->nc,
                                          e->d_ccoef + 2 * e->nc, x, abc, reinterpret_cast<double2*>(cur_dev));
  LAUNCHED();
  int st[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (st[0]) return fail(e, NECGPU_ERR_CUDA, "solve_noalloc: triangular sweep gave up waiting on a block");
  e->stats.refine_iters = iters;
  e->stats.refine_residual = rel;
  return NECGPU_OK;
}

}  // extern "C"
