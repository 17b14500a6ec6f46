// batch.cu - many cases of uneven size in one persistent launch per RK stage.
//
// A batch groups solver objects (each with its own grid, geometry and state) on one device.
// A device table holds, per case, its TMA maps, stage constants, state buffers and tile
// counts; tiles of all cases are numbered consecutively (largest cases first).  The stage
// kernel is persistent: a grid of (SM count x CTAs per SM) CTAs pulls tile numbers from a
// global counter and runs the same tile as the single-case kernel: the TMA tile
// (stage_tma.cuh, three CTAs per SM) for solvers on KERNEL_TMA, the paired-cell tile
// (stage_pair.cuh, two CTAs per SM) for solvers on KERNEL_PAIR.  A tile's stage constants
// are copied from the case table into shared memory, where the tile reads them as the
// single-case kernel reads its kernel parameters, instead of holding them in registers.
// The last CTA to find the queue empty resets the counter, so the four launches of two
// SSP-RK2 iterations are captured once in a CUDA graph and replayed; buffer roles alternate
// with the iteration's parity (Q and B swap every iteration, as in src/air_cfd.js:256).
// The autotuner times candidate z-run lengths per tile and CTA counts on the real batch
// (state saved and restored around the trials) and keeps the fastest.
//
// Mode 1 (the default) runs no persistent kernel: each case's own single-case stage launches,
// each case on a stream forked from the batch stream, are captured for two iterations in one
// CUDA graph whose per-case branches the GPU runs concurrently - small cases fill the SMs that
// large cases leave idle, and each case computes exactly what it computes alone.
#include <algorithm>
#include <numeric>
#include <vector>
#include "stage_pair.cuh"
#include "stage_tma.cuh"

namespace a3d {

namespace {

constexpr int TILE_TMA = 0, TILE_PAIR = 1;

struct __align__(128) BatchCase {
  CUtensorMap tmQ[3];  // maps over the case's three state buffers
  CUtensorMap tmC;     // map over its codes
  StageArgs a;         // stage constants (pointers, dims, far-field/fixed states, cfl, order)
  float* buf[3];
  int iQ, iS1, iB;     // buffer roles at the start of the batch step
  int nbx, nby, nbz, kz;
  long long tile_begin;
};

// Error record of a batch launch: [0] set once a tile's bounded wait ran out, [1] its table row,
// [2] its tile number, [3] how many tiles the CTA had finished before it.
constexpr int kErrWords = 4;

template <bool STAGE2, int TILE>
__device__ __forceinline__ void batch_loop(unsigned char* smem_raw, const BatchCase* __restrict__ cases, int ncases,
                                           long long total, int parity, unsigned long long* counter,
                                           long long* err) {
  __shared__ long long s_w, s_done;  // ticket; tiles this CTA finished (kept out of registers)
  __shared__ int s_failed;
  __shared__ StageArgs s_a;          // stage constants of the current tile's case
  if (threadIdx.x == 0) { s_done = 0; s_failed = 0; }
  for (;;) {
    if (threadIdx.x == 0) s_w = (long long)atomicAdd(counter, 1ULL);
    __syncthreads();
    const long long w = s_w;
    __syncthreads();
    if (w >= total) {
      // every CTA takes exactly one ticket past the end (a CTA whose tile failed keeps taking
      // tickets without work), so the last one can reset the queue for the next launch
      if (threadIdx.x == 0 && w == total + (long long)gridDim.x - 1) *counter = 0ULL;
      return;
    }
    if (s_failed) continue;
    int lo = 0, hi = ncases - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cases[mid].tile_begin <= w) lo = mid; else hi = mid - 1;
    }
    const BatchCase& C = cases[lo];
    const long long t = w - C.tile_begin;
    const int bx = (int)(t % C.nbx), by = (int)((t / C.nbx) % C.nby), bz = (int)(t / ((long long)C.nbx * C.nby));
    const int iq = parity ? C.iB : C.iQ, ib = parity ? C.iQ : C.iB;
    // stage 1: S1 = Q + dt R(Q); stage 2: B = Q/2 + (S1 + dt R(S1))/2
    const int qin = STAGE2 ? C.iS1 : iq;
    float* out = STAGE2 ? C.buf[ib] : C.buf[C.iS1];
    // Every thread of the CTA is past the previous tile (the two ticket barriers above), so
    // thread 0 may overwrite the constants; the barrier after the copy publishes them before
    // any thread reads them (a tile reads its dimensions and spacing arrays before its own
    // opening barrier).
    if (threadIdx.x == 0) s_a = C.a;
    __syncthreads();
    const bool ok = TILE == TILE_TMA
                        ? tma::stage_tile<STAGE2, true>(*reinterpret_cast<tma::TmaSmem*>(smem_raw), &C.tmQ[qin], &C.tmC,
                                                        s_a, C.buf[iq], out, bx, by, bz, C.kz)
                        : pair::stage_tile<STAGE2, true>(*reinterpret_cast<pair::PairSmem*>(smem_raw), &C.tmQ[qin],
                                                         &C.tmC, s_a, C.buf[iq], out, bx, by, bz, C.kz);
    if (!ok) {
      if (threadIdx.x == 0) {
        s_failed = 1;
        if (atomicCAS((unsigned long long*)err, 0ULL, 1ULL) == 0ULL) {
          err[1] = lo;
          err[2] = w;
          err[3] = s_done;
        }
      }
      continue;
    }
    if (threadIdx.x == 0) s_done++;
  }
}

template <bool STAGE2>
__global__ void __launch_bounds__(ring::TX * ring::TY, 3)
    k_batch_tma(const BatchCase* __restrict__ cases, int ncases, long long total, int parity,
                unsigned long long* counter, long long* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  batch_loop<STAGE2, TILE_TMA>(smem_raw, cases, ncases, total, parity, counter, err);
}

template <bool STAGE2>
__global__ void __launch_bounds__(pair::NT, 2)
    k_batch_pair(const BatchCase* __restrict__ cases, int ncases, long long total, int parity,
                 unsigned long long* counter, long long* err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  batch_loop<STAGE2, TILE_PAIR>(smem_raw, cases, ncases, total, parity, counter, err);
}

}  // namespace

}  // namespace a3d

struct a3d_batch {
  int device = 0;
  int n_sm = 148;
  cudaStream_t st = nullptr;
  std::vector<a3d_solver*> solvers;
  std::vector<cudaEvent_t> ev_in;  // one per solver: its stream's work before the batch
  cudaEvent_t ev_out = nullptr;
  a3d::BatchCase* d_cases = nullptr;
  std::vector<a3d::BatchCase> h_cases;
  std::vector<int> order;          // solver index of each table row (largest first)
  unsigned long long* d_counters = nullptr;
  long long* d_err = nullptr;      // error record of the stage launches (kErrWords words)
  long long total = 0;
  int kz = 32;
  int ctas_per_sm = 2;
  bool tma_tile = true;            // TMA tile (KERNEL_TMA solvers) or paired-cell tile (KERNEL_PAIR)
  cudaGraphExec_t graph = nullptr;
  bool table_dirty = true;
  // mode 1: every case's own single-case stage launches, each case on its own forked stream,
  // two iterations captured in one CUDA graph whose branches run concurrently
  int mode = 1;
  cudaGraphExec_t sgraph = nullptr;
  bool sgraph_dirty = true;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  // what each solver looked like when the table and the graphs were built: buffer roles, stage
  // kernel and z run, scheme constants (a solver stepped or reconfigured on its own since
  // then makes the batch rebuild them)
  std::vector<std::vector<double>> sig;
};

namespace a3d {

namespace {

void free_graph(a3d_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  if (b->sgraph) cudaGraphExecDestroy(b->sgraph);
  b->sgraph = nullptr;
  b->sgraph_dirty = true;
}

int build_table(a3d_batch* b) {
  const int n = (int)b->solvers.size();
  b->h_cases.assign(n, BatchCase{});
  long long tile = 0;
  for (int r = 0; r < n; r++) {
    a3d_solver* s = b->solvers[b->order[r]];
    BatchCase& C = b->h_cases[r];
    const bool pt = !b->tma_tile;  // the paired tile's maps have its 32 x 16-column boxes
    for (int k = 0; k < 3; k++) C.tmQ[k] = pt ? s->tmQp[k] : s->tmQ[k];
    C.tmC = pt ? s->tmCp : s->tmC;
    const int TX = 32, TY = pt ? pair::TY : ring::TY;
    fill_stage_args(s, C.a, nullptr, nullptr, nullptr, 0.5f, 0.5f);
    for (int k = 0; k < 3; k++) C.buf[k] = s->buf[k];
    C.iQ = s->iQ; C.iS1 = s->iS1; C.iB = s->iB;
    C.kz = std::max(1, std::min(b->kz, s->grid.NZ));
    C.nbx = (s->grid.NX + TX - 1) / TX;
    C.nby = (s->grid.NY + TY - 1) / TY;
    C.nbz = (s->grid.NZ + C.kz - 1) / C.kz;
    C.tile_begin = tile;
    tile += (long long)C.nbx * C.nby * C.nbz;
  }
  b->total = tile;
  A3D_CUDA(cudaMemcpyAsync(b->d_cases, b->h_cases.data(), n * sizeof(BatchCase), cudaMemcpyHostToDevice, b->st));
  b->table_dirty = false;
  return A3D_OK;
}

// The two persistent stage launches of one iteration (buffer roles of the given parity).
int launch_iteration(a3d_batch* b, int parity, cudaStream_t st) {
  const int grid = b->n_sm * b->ctas_per_sm, n = (int)b->solvers.size();
  unsigned long long* c0 = b->d_counters + 2 * parity;
  if (b->tma_tile) {
    const size_t smem = tma_smem_bytes();
    const int nt = ring::TX * ring::TY;
    k_batch_tma<false><<<grid, nt, smem, st>>>(b->d_cases, n, b->total, parity, c0, b->d_err);
    k_batch_tma<true><<<grid, nt, smem, st>>>(b->d_cases, n, b->total, parity, c0 + 1, b->d_err);
  } else {
    const size_t smem = pair_smem_bytes();
    k_batch_pair<false><<<grid, pair::NT, smem, st>>>(b->d_cases, n, b->total, parity, c0, b->d_err);
    k_batch_pair<true><<<grid, pair::NT, smem, st>>>(b->d_cases, n, b->total, parity, c0 + 1, b->d_err);
  }
  A3D_CUDA(cudaGetLastError());
  return A3D_OK;
}

// Graph of two iterations (parities 0 and 1): four persistent launches.
int build_graph(a3d_batch* b) {
  free_graph(b);
  cudaGraph_t g = nullptr;
  A3D_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  int rc = launch_iteration(b, 0, b->st);
  if (rc == A3D_OK) rc = launch_iteration(b, 1, b->st);
  cudaError_t e = cudaStreamEndCapture(b->st, &g);
  if (rc != A3D_OK) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) { set_error("graph capture: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_error("graph instantiate: %s", cudaGetErrorString(e)); return A3D_ERR_CUDA; }
  return A3D_OK;
}

std::vector<double> signature(const a3d_solver* s) {
  std::vector<double> v = {(double)s->iQ, (double)s->iS1, (double)s->iB, (double)s->kernel, (double)s->march_kz,
                           (double)s->order, s->cfl};
  v.insert(v.end(), s->F, s->F + 5);
  for (int f = 0; f < 3; f++) v.insert(v.end(), s->fix[f], s->fix[f] + 5);
  return v;
}

// Mode 1: two iterations of every case with its own stage kernel, captured from its own stream
// forked off the batch stream, so that the graph's per-case branches run concurrently.  Each
// case's arithmetic is exactly its single-case step.
int build_stream_graph(a3d_batch* b) {
  if (b->sgraph) cudaGraphExecDestroy(b->sgraph);
  b->sgraph = nullptr;
  cudaGraph_t g = nullptr;
  A3D_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  int rc = A3D_OK;
  auto cu = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == A3D_OK) { set_error("stream graph: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
  };
  cu(cudaEventRecord(b->ev_fork, b->st));
  for (size_t k = 0; k < b->solvers.size() && rc == A3D_OK; k++) {
    a3d_solver* s = b->solvers[k];
    cu(cudaStreamWaitEvent(s->st, b->ev_fork, 0));
    int iQ = s->iQ, iB = s->iB;
    const int iS1 = s->iS1;
    StageArgs a1, a2;
    for (int it = 0; it < 2 && rc == A3D_OK; it++) {  // as a3d_solver_step, on local roles
      float *Q = s->buf[iQ], *S1 = s->buf[iS1], *B = s->buf[iB];
      fill_stage_args(s, a1, Q, Q, S1, 0.f, 1.f);
      rc = launch_stage(s, a1);
      if (rc == A3D_OK) {
        fill_stage_args(s, a2, S1, Q, B, 0.5f, 0.5f);
        rc = launch_stage(s, a2);
      }
      std::swap(iQ, iB);
    }
    cu(cudaEventRecord(b->ev_join[k], s->st));
    cu(cudaStreamWaitEvent(b->st, b->ev_join[k], 0));
  }
  const cudaError_t e = cudaStreamEndCapture(b->st, &g);  // always end the capture
  if (rc != A3D_OK || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (rc == A3D_OK) { set_error("stream graph capture: %s", cudaGetErrorString(e)); rc = A3D_ERR_CUDA; }
    return rc;
  }
  const cudaError_t e2 = cudaGraphInstantiate(&b->sgraph, g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) { set_error("stream graph instantiate: %s", cudaGetErrorString(e2)); return A3D_ERR_CUDA; }
  b->sgraph_dirty = false;
  return A3D_OK;
}

int run_streams(a3d_batch* b, int n) {
  if (b->sgraph_dirty || !b->sgraph) A3D_TRY(build_stream_graph(b));
  for (int p = 0; p + 1 < n; p += 2) A3D_CUDA(cudaGraphLaunch(b->sgraph, b->st));
  A3D_CUDA(cudaEventRecord(b->ev_out, b->st));
  for (size_t k = 0; k < b->solvers.size(); k++) {
    a3d_solver* s = b->solvers[k];
    A3D_CUDA(cudaStreamWaitEvent(s->st, b->ev_out, 0));
    s->it += n & ~1;
    if (n & 1) {  // the odd iteration on the case's own stream, then back into the batch stream
      A3D_TRY(a3d_solver_step(s, 1));
      A3D_CUDA(cudaEventRecord(b->ev_in[k], s->st));
      A3D_CUDA(cudaStreamWaitEvent(b->st, b->ev_in[k], 0));
    }
  }
  if (n & 1) {  // buffer roles moved on
    b->sgraph_dirty = true;
    for (size_t k = 0; k < b->solvers.size(); k++) b->sig[k] = signature(b->solvers[k]);
  }
  return A3D_OK;
}

// Runs n iterations of every case; updates each solver's roles and iteration count.
int run(a3d_batch* b, int n) {
  bool changed = b->sig.size() != b->solvers.size();
  if (!changed)
    for (size_t k = 0; k < b->solvers.size() && !changed; k++) changed = signature(b->solvers[k]) != b->sig[k];
  if (changed) {
    b->table_dirty = true;
    b->sgraph_dirty = true;
    b->sig.clear();
    for (a3d_solver* s : b->solvers) b->sig.push_back(signature(s));
  }
  for (size_t k = 0; k < b->solvers.size(); k++) {  // order after each solver's own work
    A3D_CUDA(cudaEventRecord(b->ev_in[k], b->solvers[k]->st));
    A3D_CUDA(cudaStreamWaitEvent(b->st, b->ev_in[k], 0));
  }
  if (b->mode == 1) return run_streams(b, n);
  if (b->table_dirty) A3D_TRY(build_table(b));
  if (!b->graph) A3D_TRY(build_graph(b));
  for (int p = 0; p + 1 < n; p += 2) A3D_CUDA(cudaGraphLaunch(b->graph, b->st));
  if (n & 1) A3D_TRY(launch_iteration(b, 0, b->st));
  A3D_CUDA(cudaEventRecord(b->ev_out, b->st));
  for (a3d_solver* s : b->solvers) {
    A3D_CUDA(cudaStreamWaitEvent(s->st, b->ev_out, 0));
    if (n & 1) std::swap(s->iQ, s->iB);
    s->it += n;
  }
  if (n & 1) {
    b->table_dirty = true;
    for (size_t k = 0; k < b->solvers.size(); k++) b->sig[k] = signature(b->solvers[k]);
  }
  return A3D_OK;
}

}  // namespace

}  // namespace a3d

using namespace a3d;

extern "C" int a3d_batch_create(a3d_solver* const* solvers, int32_t n, a3d_batch** out) {
  clear_error();
  A3D_ARG(solvers && out && n >= 1, "solvers");
  const int dev = solvers[0]->device;
  for (int k = 0; k < n; k++) {
    A3D_ARG(solvers[k], "null solver");
    A3D_ARG(solvers[k]->device == dev, "all solvers of a batch must live on one device");
    A3D_ARG(solvers[k]->own_k0 == 0 && solvers[k]->own_k1 == solvers[k]->grid.NZ && !solvers[k]->nbr[0] &&
                !solvers[k]->nbr[1],
            "z-slab solvers cannot be batched");
    A3D_ARG(solvers[k]->kernel == KERNEL_PAIR || solvers[k]->kernel == KERNEL_TMA,
            "batch needs solvers on a TMA tile (stage kernel 2 or 4)");
    A3D_ARG(solvers[k]->kernel == solvers[0]->kernel, "all solvers of a batch must select the same stage kernel");
  }
  A3D_CUDA(cudaSetDevice(dev));
  a3d_batch* b = new a3d_batch();
  b->device = dev;
  b->tma_tile = solvers[0]->kernel == KERNEL_TMA;
  b->ctas_per_sm = b->tma_tile ? 3 : 2;
  cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, dev);
  b->solvers.assign(solvers, solvers + n);
  b->order.resize(n);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return b->solvers[x]->N > b->solvers[y]->N; });
  int rc = A3D_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming);
  b->ev_in.assign(n, nullptr);
  for (int k = 0; k < n && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&b->ev_in[k], cudaEventDisableTiming);
  b->ev_join.assign(n, nullptr);
  for (int k = 0; k < n && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_cases, (size_t)n * sizeof(BatchCase));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_counters, 8 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counters, 0, 8 * sizeof(unsigned long long), b->st);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_err, kErrWords * sizeof(long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_err, 0, kErrWords * sizeof(long long), b->st);
  if (e != cudaSuccess) { set_error("batch setup: %s", cudaGetErrorString(e)); rc = e == cudaErrorMemoryAllocation ? A3D_ERR_NOMEM : A3D_ERR_CUDA; }
  if (rc == A3D_OK) {
    const int pt = (int)pair_smem_bytes(), tt = (int)tma_smem_bytes();
    int r = cudaFuncSetAttribute(k_batch_pair<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, pt);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_pair<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, pt);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_pair<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_pair<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tt);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tt);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_tma<false>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_batch_tma<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (r != cudaSuccess) { set_error("batch kernel attributes: %s", cudaGetErrorString((cudaError_t)r)); rc = A3D_ERR_CUDA; }
  }
  if (rc != A3D_OK) { a3d_batch_destroy(b); return rc; }
  *out = b;
  return A3D_OK;
}

extern "C" int a3d_batch_destroy(a3d_batch* b) {
  if (!b) return A3D_OK;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  free_graph(b);
  cudaFree(b->d_cases);
  cudaFree(b->d_counters);
  cudaFree(b->d_err);
  for (cudaEvent_t e : b->ev_in) if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : b->ev_join) if (e) cudaEventDestroy(e);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return A3D_OK;
}

extern "C" int a3d_batch_set_mode(a3d_batch* b, int32_t mode) {
  clear_error();
  A3D_ARG(b, "null batch");
  A3D_ARG(mode == 0 || mode == 1, "batch mode");
  b->mode = mode;
  return A3D_OK;
}

extern "C" int a3d_batch_get_mode(a3d_batch* b, int32_t* mode) {
  clear_error();
  A3D_ARG(b && mode, "null pointer");
  *mode = b->mode;
  return A3D_OK;
}

extern "C" int a3d_batch_set_schedule(a3d_batch* b, int32_t kz, int32_t ctas_per_sm) {
  clear_error();
  A3D_ARG(b, "null batch");
  A3D_ARG(kz >= 1 && kz <= 1024 && ctas_per_sm >= 1 && ctas_per_sm <= (b->tma_tile ? 3 : 2), "schedule");
  b->kz = kz;
  b->ctas_per_sm = ctas_per_sm;
  b->table_dirty = true;
  free_graph(b);
  return A3D_OK;
}

extern "C" int a3d_batch_get_schedule(a3d_batch* b, int32_t* kz, int32_t* ctas_per_sm, int64_t* tiles) {
  clear_error();
  A3D_ARG(b, "null batch");
  if (kz) *kz = b->kz;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  if (tiles) *tiles = b->total;
  return A3D_OK;
}

extern "C" int a3d_batch_step(a3d_batch* b, int32_t n) {
  clear_error();
  A3D_ARG(b && n >= 0, "batch step");
  A3D_CUDA(cudaSetDevice(b->device));
  return run(b, n);
}

extern "C" int a3d_batch_sync(a3d_batch* b) {
  clear_error();
  A3D_ARG(b, "null batch");
  A3D_CUDA(cudaSetDevice(b->device));
  A3D_CUDA(cudaStreamSynchronize(b->st));
  long long rec[kErrWords];
  A3D_CUDA(cudaMemcpy(rec, b->d_err, sizeof(rec), cudaMemcpyDeviceToHost));
  if (rec[0]) {
    // clear the record (the queues were reset by the launches themselves) and report; the
    // failed case keeps its own flag, so its solver reports the timeout until it is rebuilt
    A3D_CUDA(cudaMemset(b->d_err, 0, sizeof(rec)));
    const int row = (int)rec[1];
    const a3d_solver* s = b->solvers[b->order[row]];
    set_error("batch stage: a bounded wait ran out in case %d (%dx%dx%d cells), tile %lld, after %lld tiles on "
              "that CTA", b->order[row], s->grid.NX, s->grid.NY, s->grid.NZ, rec[2] - b->h_cases[row].tile_begin,
              rec[3]);
    return A3D_ERR_TIMEOUT;
  }
  for (a3d_solver* s : b->solvers) A3D_TRY(check_kernel_error(s));
  return A3D_OK;
}

extern "C" int a3d_batch_tune(a3d_batch* b, int32_t trial_iters, int32_t* best_kz, int32_t* best_ctas,
                              float* best_ms) {
  clear_error();
  A3D_ARG(b && trial_iters >= 2, "tune");
  A3D_CUDA(cudaSetDevice(b->device));
  const int n = (int)b->solvers.size();
  const int it = trial_iters & ~1;  // even: the buffer roles come back to where they were
  // save every case's current state and iteration count
  std::vector<float*> saved(n, nullptr);
  std::vector<long> saved_it(n);
  int rc = A3D_OK;
  for (int k = 0; k < n && rc == A3D_OK; k++) {
    a3d_solver* s = b->solvers[k];
    A3D_CUDA(cudaStreamSynchronize(s->st));
    if (cudaMalloc(&saved[k], 5 * s->Np * sizeof(float)) != cudaSuccess) { set_error("tune: no memory for the state copy"); rc = A3D_ERR_NOMEM; break; }
    A3D_CUDA(cudaMemcpyAsync(saved[k], s->buf[s->iQ], 5 * s->Np * sizeof(float), cudaMemcpyDeviceToDevice, s->st));
    saved_it[k] = s->it;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int bkz = b->kz, bct = b->ctas_per_sm;
  const int kzs[] = {8, 16, 32, 64};
  const int max_ct = b->tma_tile ? 3 : 2;
  b->mode = 0;
  for (int ct = 1; ct <= max_ct && rc == A3D_OK; ct++)
    for (int kz : kzs) {
      if (rc != A3D_OK) break;
      a3d_batch_set_schedule(b, kz, ct);
      rc = run(b, 2);  // warm: builds the table and the graph
      if (rc != A3D_OK) break;
      cudaEventRecord(e0, b->st);
      rc = run(b, it);
      cudaEventRecord(e1, b->st);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) { best = ms; bkz = kz; bct = ct; }
    }
  if (rc == A3D_OK) rc = a3d_batch_set_schedule(b, bkz, bct);
  int bmode = 0;
  if (rc == A3D_OK) {  // the concurrent stream graph of single-case launches
    b->mode = 1;
    rc = run(b, 2);
    if (rc == A3D_OK) {
      cudaEventRecord(e0, b->st);
      rc = run(b, it);
      cudaEventRecord(e1, b->st);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) { best = ms; bmode = 1; }
    }
    b->mode = bmode;
  }
  for (int k = 0; k < n; k++) {  // restore
    a3d_solver* s = b->solvers[k];
    cudaStreamSynchronize(b->st);
    if (saved[k]) {
      cudaMemcpy(s->buf[s->iQ], saved[k], 5 * s->Np * sizeof(float), cudaMemcpyDeviceToDevice);
      cudaFree(saved[k]);
    }
    s->it = saved_it[k];
  }
  b->table_dirty = true;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_kz) *best_kz = bkz;
  if (best_ctas) *best_ctas = bct;
  if (best_ms) *best_ms = best / (float)it;
  return rc;
}
