// Batched D2Q4x6 step: many independent problems (geometries, load cases,
// uneven lattice sizes) advanced together.  Included at the end of
// cvlbm2d.cu; reuses the fused tile body (fused2_tile) and the cooperative
// link body (link2_block).
//
// Per lattice step three launches cover every instance:
//   k_batch_nodes2   persistent: a grid of (SMs x resident blocks) walks the
//                    work list of (instance, tile) pairs
//   k_batch_links2   persistent: walks (instance, 16-link group) pairs
//   k_batch_tick2    advances each active instance's clock and step counter
// Every `check_every` steps the node kernel also stores U and u of every
// active node, k_batch_partial2 reduces |u - u_prev|^2 and |u|^2 per
// (instance, tile) in a fixed order (u_prev = u at the previous check) and
// k_batch_residual2 retires instances whose residual
// |u - u_prev|_2 / (check_every * |u|_2), the relative displacement change per
// step, fell below the tolerance (after a minimum time, e.g. the end of a load
// ramp).  The velocity moment is no measure of convergence here: with the
// displacement sweep the damped steady state keeps a small constant v whose
// increments the sweep cancels every step.  Retired instances' work items
// return at once.  The whole step sequence is captured in one CUDA graph
// (cvlbm2d_batch_graph_create).
//
// Each instance keeps its own population and u* ping-pong; the buffer that
// holds the current state is selected by the parity of the steps the instance
// has taken inside the batch.
#pragma once

#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct Inst2 {
  Ctx2 c;
  const uint8_t* need;
  const int32_t* partner;
  double* scratch;
  double* f[2];   // population buffers; f[par] holds the current state
  double* us[2];  // u* buffers
  double* U;
  double* u;
  double* u_prev;  // [2*N] u at the previous residual check (batch-owned)
  int* invalid;
};

struct InstState2 {
  long long step;       // step index of the instance (interval tests)
  long long base;       // step index at batch creation (buffer parity)
  double clock;         // device time
  double residual;      // last residual, -1 before the second check
  int active;           // 1 while stepping
  int status;           // 0 running, 1 converged, -1 invalid state
  int checks;           // residual checks done
  int pad;
};

__device__ __forceinline__ int parity_of(const InstState2& s) { return (int)((s.step - s.base) & 1); }

template <int TY, int MINB>
__global__ void __launch_bounds__(kTX * TY, MINB)
    k_batch_nodes2(const Inst2* __restrict__ inst, InstState2* __restrict__ st,
                   const int2* __restrict__ work, int n_work, int store_all) {
  extern __shared__ double smem2[];
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    __syncthreads();  // the previous item's phase C still reads shared memory
    const int2 wk = work[w];
    if (!st[wk.x].active) continue;
    const Inst2& I = inst[wk.x];
    const long long step = st[wk.x].step;
    const int par = parity_of(st[wk.x]);
    const cvlbm2d_problem& p = I.c.p;
    const int sweep = p.disp_interval > 0 && step % p.disp_interval == 0;
    const int repair = p.rep_interval > 0 && step % p.rep_interval == 0;
    Fused2 fz{nullptr, 0, p.tiles_j, I.need, I.partner, I.scratch, store_all};
    fused2_tile<TY, false>(I.c, fz, wk.y, I.f[par], I.f[par ^ 1], I.U, I.u, I.us[par], I.us[par ^ 1],
                    I.invalid, &st[wk.x].clock, 0.0, sweep, repair, smem2);
  }
}

// The batched link kernel runs 8 lanes per link (16 links per block): in the
// batch the link work is throughput-bound, so twice the links in flight per
// SM pay for each link's longer gather.
constexpr int kBatchLG = 8;
constexpr int kBatchLinksPerBlock = kLinkThreads2 / kBatchLG;

template <int MAT, int RECON = -1, int SOLVER = -1>
__global__ void __launch_bounds__(kLinkThreads2, 3)
    k_batch_links2(const Inst2* __restrict__ inst, const InstState2* __restrict__ st,
                   const int2* __restrict__ work, int n_work) {
  __shared__ LinkShared2 sh[kBatchLinksPerBlock];
  __shared__ LinkBC2 bc;
  const int lane = threadIdx.x & (kBatchLG - 1);
  const int grp = threadIdx.x / kBatchLG;
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    const int2 wk = work[w];
    // uniform over the block (one work item per iteration): the barriers
    // below are reached by every thread or by none
    if (!st[wk.x].active) continue;
    const Inst2& I = inst[wk.x];
    __syncthreads();  // the previous item's readers of bc are done (link2_group restages it)
    double* f1 = I.f[parity_of(st[wk.x]) ^ 1];
    const Mat m = link_mat2<MAT>(I.c);
    link2_group<RECON, SOLVER, kBatchLG>(I.c, m, bc, sh[grp], lane, wk.y + grp, f1, f1, I.U, I.u,
                               &st[wk.x].clock, 0.0,
                0.5 * I.c.p.dt, 1, I.scratch, I.partner);
  }
}

// Instances [i0, i1).
__global__ void k_batch_tick2(const Inst2* __restrict__ inst, InstState2* __restrict__ st, int i0,
                              int i1) {
  const int i = i0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= i1 || !st[i].active) return;
  st[i].clock = st[i].clock + inst[i].c.p.dt;
  st[i].step = st[i].step + 1;
  if (*inst[i].invalid) {  // non-positive Jacobian: stop this instance, keep the others
    st[i].active = 0;
    st[i].status = -1;
  }
}

// Per (instance, tile): sum of |u - u_prev|^2 and |u|^2 over the tile's
// active nodes, reduced in a fixed order (deterministic for a given tile
// height); u_prev is then replaced by u.
template <int TY>
__global__ void __launch_bounds__(kTX * TY)
    k_batch_partial2(const Inst2* __restrict__ inst, const InstState2* __restrict__ st,
                     const int2* __restrict__ work, int n_work, double2* __restrict__ partial) {
  __shared__ double sv[kTX * TY], su[kTX * TY];
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    __syncthreads();
    const int2 wk = work[w];
    const Inst2& I = inst[wk.x];
    const cvlbm2d_problem& p = I.c.p;
    const int N = I.c.N;
    const int i = (wk.y / p.tiles_j) * TY + (int)(threadIdx.x >> 5);
    const int j = (wk.y % p.tiles_j) * kTX + (int)(threadIdx.x & 31);
    double v2 = 0.0, u2 = 0.0;
    if (st[wk.x].active && i < p.nx && j < p.ny && p.active[i * p.ny + j]) {
      const int n = i * p.ny + j;
      const double u0 = I.u[n], u1 = I.u[(size_t)N + n];
      const double d0 = u0 - I.u_prev[n], d1 = u1 - I.u_prev[(size_t)N + n];
      v2 = d0 * d0 + d1 * d1;
      u2 = u0 * u0 + u1 * u1;
      I.u_prev[n] = u0;
      I.u_prev[(size_t)N + n] = u1;
    }
    sv[threadIdx.x] = v2;
    su[threadIdx.x] = u2;
    __syncthreads();
    for (int h = (kTX * TY) / 2; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) {
        sv[threadIdx.x] += sv[threadIdx.x + h];
        su[threadIdx.x] += su[threadIdx.x + h];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[w] = make_double2(sv[0], su[0]);
  }
}

__global__ void k_batch_residual2(const Inst2* __restrict__ inst, InstState2* __restrict__ st,
                                  const int* __restrict__ work_start,
                                  const double2* __restrict__ partial, int n, double tol,
                                  double t_min, int interval) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !st[i].active) return;
  double sv = 0.0, su = 0.0;
  for (int w = work_start[i]; w < work_start[i + 1]; ++w) {
    sv += partial[w].x;
    su += partial[w].y;
  }
  const double r = su > 0.0 ? sqrt(sv) / ((double)interval * sqrt(su)) : (sv > 0.0 ? 1.0 : 0.0);
  st[i].checks = st[i].checks + 1;
  if (st[i].checks < 2) return;  // no earlier displacement to compare with
  st[i].residual = r;
  if (st[i].clock >= t_min && r < tol) {
    st[i].active = 0;
    st[i].status = 1;
  }
}

using BatchNodesFn = void (*)(const Inst2*, InstState2*, const int2*, int, int);
using BatchPartialFn = void (*)(const Inst2*, const InstState2*, const int2*, int, double2*);

struct BatchVariant2 {
  BatchNodesFn nodes;
  BatchPartialFn partial;
  int threads;
  size_t smem;
  int tile_i;
};

BatchVariant2 batch_variant(int v) {
  switch (v) {
    case 1: return {k_batch_nodes2<8, 2>, k_batch_partial2<8>, kTX * 8, fused_smem2<8>(), 8};
    case 2: return {k_batch_nodes2<8, 3>, k_batch_partial2<8>, kTX * 8, fused_smem2<8>(), 8};
    case 3: return {k_batch_nodes2<16, 2>, k_batch_partial2<16>, kTX * 16, fused_smem2<16>(), 16};
    case 4: return {k_batch_nodes2<4, 4>, k_batch_partial2<4>, kTX * 4, fused_smem2<4>(), 4};
    default: return {k_batch_nodes2<16, 1>, k_batch_partial2<16>, kTX * 16, fused_smem2<16>(), 16};
  }
}

}  // namespace

struct cvlbm2d_batch {
  int n_inst = 0;
  int variant = 0;
  int node_grid = 0, link_grid = 0;
  int n_work = 0, n_lwork = 0;
  Inst2* d_inst = nullptr;
  InstState2* d_state = nullptr;
  int2* d_work = nullptr;
  int2* d_lwork = nullptr;
  int* d_work_start = nullptr;
  double* d_uprev = nullptr;
  double2* d_partial = nullptr;
  // two instance groups on two streams (see batch_run_grouped)
  int groups = 1;
  int inst_split = 0, work_split = 0, lwork_split = 0;
  int all_neo_hooke = 0;  // every instance neo-Hooke: the link kernel compiled for it
  int local_f_solver = -1;  // ... and every one local_f with this Neumann solver
  cudaStream_t side = nullptr;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
};

namespace {

void batch_free(cvlbm2d_batch* b) {
  if (!b) return;
  cudaFree(b->d_inst);
  cudaFree(b->d_state);
  cudaFree(b->d_work);
  cudaFree(b->d_lwork);
  cudaFree(b->d_work_start);
  cudaFree(b->d_partial);
  cudaFree(b->d_uprev);
  if (b->ev_a) cudaEventDestroy(b->ev_a);
  if (b->ev_b) cudaEventDestroy(b->ev_b);
  if (b->side) cudaStreamDestroy(b->side);
  delete b;
}

// Node work items [w0, w1), link items [l0, l1), instances [i0, i1).
void batch_nodes(cvlbm2d_batch* b, int w0, int w1, int store_all, cudaStream_t s) {
  if (w1 <= w0) return;
  const BatchVariant2 v = batch_variant(b->variant);
  const int grid = b->node_grid < w1 - w0 ? b->node_grid : w1 - w0;
  v.nodes<<<grid, v.threads, v.smem, s>>>(b->d_inst, b->d_state, b->d_work + w0, w1 - w0,
                                          store_all);
  cv::count_launches(1);
}

// The link kernel build for the batch: fixed at compile time to the law, the
// closure and the Neumann solver when every instance shares them.
using BatchLinkFn = void (*)(const Inst2*, const InstState2*, const int2*, int);
BatchLinkFn batch_link_kernel(const cvlbm2d_batch* b) {
  if (!b->all_neo_hooke) return k_batch_links2<-1>;
  switch (b->local_f_solver) {
    case kSolverFD: return k_batch_links2<kMatNeoHooke, 12, kSolverFD>;
    case kSolverAcoustic: return k_batch_links2<kMatNeoHooke, 12, kSolverAcoustic>;
    case kSolverEnergy: return k_batch_links2<kMatNeoHooke, 12, kSolverEnergy>;
    default: return k_batch_links2<kMatNeoHooke>;
  }
}

void batch_links_tick(cvlbm2d_batch* b, int l0, int l1, int i0, int i1, cudaStream_t s) {
  if (l1 > l0) {
    const int grid = b->link_grid < l1 - l0 ? b->link_grid : l1 - l0;
    batch_link_kernel(b)<<<grid, kLinkThreads2, 0, s>>>(b->d_inst, b->d_state,
                                                       b->d_lwork + l0, l1 - l0);
    cv::count_launches(1);
  }
  if (i1 > i0) {
    k_batch_tick2<<<blocks(i1 - i0, 128), 128, 0, s>>>(b->d_inst, b->d_state, i0, i1);
    cv::count_launches(1);
  }
}

void batch_step(cvlbm2d_batch* b, int store_all, cudaStream_t s) {
  batch_nodes(b, 0, b->n_work, store_all, s);
  batch_links_tick(b, 0, b->n_lwork, 0, b->n_inst, s);
}

void batch_check(cvlbm2d_batch* b, int check_every, double tol, double t_min, cudaStream_t s) {
  const BatchVariant2 v = batch_variant(b->variant);
  if (b->n_work <= 0) return;
  v.partial<<<b->node_grid, v.threads, 0, s>>>(b->d_inst, b->d_state, b->d_work, b->n_work,
                                               b->d_partial);
  cv::count_launches(1);
  k_batch_residual2<<<blocks(b->n_inst, 128), 128, 0, s>>>(b->d_inst, b->d_state,
                                                           b->d_work_start, b->d_partial,
                                                           b->n_inst, tol, t_min, check_every);
  cv::count_launches(1);
}

// Two instance groups, each advanced by its own node / link / tick launches
// on its own stream (group A on the caller's stream, group B on `side`).
// The groups share no buffer and no state entry, so every instance takes
// exactly its serial sequence of launches; group B's node kernel of a step
// starts once group A's has finished, so that it runs while A's link kernel
// (a set of long per-link chains) does, and the offset carries on from step
// to step.  At residual-check steps the groups join for the check over all
// instances.
void batch_run_grouped(cvlbm2d_batch* b, int nsteps, int check_every, double tol, double t_min,
                       cudaStream_t s) {
  const int ia = b->inst_split, wa = b->work_split, la = b->lwork_split;
  cudaEventRecord(b->ev_b, s);  // the side stream starts after prior work
  cudaStreamWaitEvent(b->side, b->ev_b, 0);
  bool offset = true;
  for (int k = 0; k < nsteps; ++k) {
    const bool check = check_every > 0 && (k + 1) % check_every == 0;
    // an attached kernel timer brackets group A's node launch (group B's
    // overlaps A's link kernel on the side stream and is not timed)
    int tk = timer_begin(s);
    batch_nodes(b, 0, wa, check ? 1 : 0, s);
    timer_end(tk, s);
    if (offset) {
      cudaEventRecord(b->ev_a, s);
      cudaStreamWaitEvent(b->side, b->ev_a, 0);
      offset = false;
    }
    batch_links_tick(b, 0, la, 0, ia, s);
    batch_nodes(b, wa, b->n_work, check ? 1 : 0, b->side);
    batch_links_tick(b, la, b->n_lwork, ia, b->n_inst, b->side);
    if (check) {
      cudaEventRecord(b->ev_b, b->side);
      cudaStreamWaitEvent(s, b->ev_b, 0);
      batch_check(b, check_every, tol, t_min, s);
      cudaEventRecord(b->ev_b, s);
      cudaStreamWaitEvent(b->side, b->ev_b, 0);
      offset = true;
    }
  }
  cudaEventRecord(b->ev_b, b->side);  // join: the run ends on the caller's stream
  cudaStreamWaitEvent(s, b->ev_b, 0);
}

}  // namespace

extern "C" int cvlbm2d_batch_create(int32_t n_inst, const cvlbm2d_problem* problems,
                                    const cvlbm2d_fields* fields, const int64_t* step0,
                                    const double* time0, int32_t tile_variant,
                                    int32_t grid_blocks, cvlbm2d_batch** out) {
  if (!out || !problems || !fields || !step0 || !time0 || n_inst <= 0)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm2d_batch_create: bad arguments");
  *out = nullptr;
  const int tile_i = cvlbm2d_tile_variant(tile_variant);
  if (tile_i <= 0 || tile_variant >= kSplitVariant)
    return fail(CVLBM_ERR_INVALID_ARG, "cvlbm2d_batch_create: unknown tile variant");
  std::vector<Inst2> hi(n_inst);
  std::vector<InstState2> hs(n_inst);
  std::vector<int2> work, lwork;
  std::vector<int> work_start(n_inst + 1, 0);
  std::vector<int> tiles;
  for (int i = 0; i < n_inst; ++i) {
    const cvlbm2d_problem* p = &problems[i];
    const cvlbm2d_fields* f = &fields[i];
    int rc = check_problem(p, f);
    if (rc) return rc;
    if (!fused_ok(p, f) || p->tile_i != tile_i)
      return fail(CVLBM_ERR_INVALID_ARG,
                  "cvlbm2d_batch_create: every instance needs the fused-step tables built for "
                  "the batch's tile variant");
    hi[i].c = make_ctx(p);
    hi[i].need = p->need_fields;
    hi[i].partner = p->link_partner;
    hi[i].scratch = f->link_scratch;
    hi[i].f[0] = f->f0;
    hi[i].f[1] = f->f1;
    hi[i].us[0] = f->u_star;
    hi[i].us[1] = f->u_next;
    hi[i].U = f->U;
    hi[i].u = f->u;
    hi[i].invalid = f->invalid;
    hs[i] = InstState2{step0[i], step0[i], time0[i], -1.0, 1, 0, 0, 0};
    tiles.resize(p->n_tiles);
    if (p->n_tiles > 0 &&
        cudaMemcpy(tiles.data(), p->tiles, sizeof(int) * p->n_tiles, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      return fail(CVLBM_ERR_CUDA, "cvlbm2d_batch_create: reading a tile list failed");
    work_start[i] = (int)work.size();
    // raster order (a solver's list may hold its inner tiles first)
    std::sort(tiles.begin(), tiles.end());
    for (int t : tiles) work.push_back(make_int2(i, t));
    for (int l = 0; l < p->n_links; l += kBatchLinksPerBlock) lwork.push_back(make_int2(i, l));
  }
  work_start[n_inst] = (int)work.size();
  cvlbm2d_batch* b = new cvlbm2d_batch();
  size_t uprev_total = 0;
  for (int i = 0; i < n_inst; ++i) uprev_total += 2 * (size_t)hi[i].c.N;
  if (cudaMalloc(&b->d_uprev, sizeof(double) * uprev_total) != cudaSuccess ||
      cudaMemset(b->d_uprev, 0, sizeof(double) * uprev_total) != cudaSuccess) {
    batch_free(b);
    return fail(CVLBM_ERR_CUDA, "cvlbm2d_batch_create: residual buffer allocation failed");
  }
  {
    size_t off = 0;
    for (int i = 0; i < n_inst; ++i) {
      hi[i].u_prev = b->d_uprev + off;
      off += 2 * (size_t)hi[i].c.N;
    }
  }
  b->n_inst = n_inst;
  b->variant = tile_variant;
  b->n_work = (int)work.size();
  b->n_lwork = (int)lwork.size();
  const BatchVariant2 v = batch_variant(tile_variant);
  cudaFuncSetAttribute(v.nodes, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem);
  int dev = 0, sms = 148, per_sm = 1, per_sm_l = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, v.nodes, v.threads, v.smem);
  b->all_neo_hooke = 1;
  b->local_f_solver = problems[0].recon == 12 ? problems[0].normal_solver : -1;
  for (int i = 0; i < n_inst; ++i) {
    if (problems[i].mat.model != kMatNeoHooke) b->all_neo_hooke = 0;
    if (problems[i].recon != 12 || problems[i].normal_solver != b->local_f_solver)
      b->local_f_solver = -1;
  }
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_l, batch_link_kernel(b), kLinkThreads2,
                                                0);
  const int full = sms * (per_sm > 0 ? per_sm : 1);
  b->node_grid = grid_blocks > 0 ? grid_blocks : full;
  if (b->node_grid > b->n_work) b->node_grid = b->n_work > 0 ? b->n_work : 1;
  b->link_grid = sms * (per_sm_l > 0 ? per_sm_l : 1);
  if (b->link_grid > b->n_lwork) b->link_grid = b->n_lwork > 0 ? b->n_lwork : 1;
  bool ok = cudaMalloc(&b->d_inst, sizeof(Inst2) * n_inst) == cudaSuccess &&
            cudaMalloc(&b->d_state, sizeof(InstState2) * n_inst) == cudaSuccess &&
            cudaMalloc(&b->d_work, sizeof(int2) * (work.size() + 1)) == cudaSuccess &&
            cudaMalloc(&b->d_lwork, sizeof(int2) * (lwork.size() + 1)) == cudaSuccess &&
            cudaMalloc(&b->d_work_start, sizeof(int) * (n_inst + 1)) == cudaSuccess &&
            cudaMalloc(&b->d_partial, sizeof(double2) * (work.size() + 1)) == cudaSuccess;
  ok = ok && cudaMemcpy(b->d_inst, hi.data(), sizeof(Inst2) * n_inst,
                        cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cudaMemcpy(b->d_state, hs.data(), sizeof(InstState2) * n_inst,
                        cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && (work.empty() || cudaMemcpy(b->d_work, work.data(), sizeof(int2) * work.size(),
                                         cudaMemcpyHostToDevice) == cudaSuccess);
  ok = ok && (lwork.empty() || cudaMemcpy(b->d_lwork, lwork.data(), sizeof(int2) * lwork.size(),
                                          cudaMemcpyHostToDevice) == cudaSuccess);
  ok = ok && cudaMemcpy(b->d_work_start, work_start.data(), sizeof(int) * (n_inst + 1),
                        cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    batch_free(b);
    return fail(CVLBM_ERR_CUDA, "cvlbm2d_batch_create: device allocation or upload failed");
  }
  // two instance groups of about equal node work (CVLBM_BATCH_GROUPS=1: one)
  const char* ge = std::getenv("CVLBM_BATCH_GROUPS");
  if (!(ge && std::strcmp(ge, "1") == 0) && n_inst > 1) {
    int split = 1;
    while (split < n_inst - 1 && work_start[split] < b->n_work / 2) ++split;
    int lsplit = 0;
    while (lsplit < b->n_lwork && lwork[lsplit].x < split) ++lsplit;
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreateWithFlags(&b->ev_a, cudaEventDisableTiming) == cudaSuccess &&
        cudaEventCreateWithFlags(&b->ev_b, cudaEventDisableTiming) == cudaSuccess) {
      b->groups = 2;
      b->inst_split = split;
      b->work_split = work_start[split];
      b->lwork_split = lsplit;
    }
  }
  *out = b;
  return CVLBM_OK;
}

extern "C" int cvlbm2d_batch_run(cvlbm2d_batch* b, int32_t nsteps, int32_t check_every,
                                 double tol, double t_min, void* stream) {
  if (!b) return fail(CVLBM_ERR_INVALID_ARG, "null batch");
  if (nsteps < 0) return fail(CVLBM_ERR_INVALID_ARG, "negative step count");
  cudaStream_t s = (cudaStream_t)stream;
  if (b->groups == 2) {
    batch_run_grouped(b, nsteps, check_every, tol, t_min, s);
    return check_launch("cvlbm2d_batch_run");
  }
  for (int k = 0; k < nsteps; ++k) {
    const bool check = check_every > 0 && (k + 1) % check_every == 0;
    int tk = timer_begin(s);
    batch_step(b, check ? 1 : 0, s);
    timer_end(tk, s);
    if (check) batch_check(b, check_every, tol, t_min, s);
  }
  return check_launch("cvlbm2d_batch_run");
}

extern "C" int cvlbm2d_batch_graph_create(cvlbm2d_batch* b, int32_t nsteps, int32_t check_every,
                                          double tol, double t_min, cvlbm_graph** out) {
  if (!b || !out) return fail(CVLBM_ERR_INVALID_ARG, "null batch or output");
  if (nsteps <= 0) return fail(CVLBM_ERR_INVALID_ARG, "nsteps must be positive");
  return capture_graph(
      [&](cudaStream_t s) { return cvlbm2d_batch_run(b, nsteps, check_every, tol, t_min, s); },
      out);
}

extern "C" int cvlbm2d_batch_status(cvlbm2d_batch* b, int32_t* active, int32_t* status,
                                    int64_t* steps, double* time, double* residual,
                                    void* stream) {
  if (!b) return fail(CVLBM_ERR_INVALID_ARG, "null batch");
  std::vector<InstState2> hs(b->n_inst);
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(hs.data(), b->d_state, sizeof(InstState2) * b->n_inst,
                      cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return fail(CVLBM_ERR_CUDA, "cvlbm2d_batch_status: copy failed");
  for (int i = 0; i < b->n_inst; ++i) {
    if (active) active[i] = hs[i].active;
    if (status) status[i] = hs[i].status;
    if (steps) steps[i] = hs[i].step;
    if (time) time[i] = hs[i].clock;
    if (residual) residual[i] = hs[i].residual;
  }
  return CVLBM_OK;
}

extern "C" int cvlbm2d_batch_launch_grid(const cvlbm2d_batch* b, int32_t* node_grid,
                                         int32_t* n_work) {
  if (!b) return fail(CVLBM_ERR_INVALID_ARG, "null batch");
  if (node_grid) *node_grid = b->node_grid;
  if (n_work) *n_work = b->n_work;
  return CVLBM_OK;
}

extern "C" void cvlbm2d_batch_destroy(cvlbm2d_batch* b) { batch_free(b); }
