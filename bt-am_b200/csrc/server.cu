// Job server: relaxation and master-equation jobs of many sizes served
// concurrently on one device (no counterpart in the reference, which runs
// one simulation per MPI job).
//
// Each job is a whole system: submitted with its host arrays (copied at
// submission), admitted by its estimated device-memory footprint
// (sched.hpp), then run by one of the worker threads on its own
// btam_system, i.e. its own CUDA stream, with q, sigma, x, the images and
// the neighbour lists resident on the device from creation to the last step.
// A job that arrives while others run starts as soon as a worker slot and
// its memory are free.
//
// Continuous batching: the residual evaluations of all running jobs of up
// to kBatchMaxSites sites go through one batcher (EvalBatcher below); larger
// jobs run their own kernels on their own streams, overlapping with the
// rounds.  A job's solver (L-BFGS steps,
// master-equation steps) runs on its own thread and stream as before; each
// time it needs an evaluation it hands its system to the batcher and waits.
// The batcher collects the requests of every running job (or those that
// arrive within a short window), copies their states into one batch layout
// (batch.cu: every job's sites renumbered into one device layout, rebuilt
// when a job joins), evaluates them all with one set of launches, and copies
// each job's results back into its own buffers; the job's stream waits for
// that and carries on.  So the jobs in flight share every evaluation launch
// instead of each launching its own kernels, and a job's results are the
// same alone and in the mix (every kernel is deterministic, a system's rows
// never mix with another's, and the batch's kernel shapes are fixed).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/btam.h"
#include "adp_kernels.cuh"
#include "internal.cuh"
#include "sched.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  long long id = 0;
  btam_job_spec spec{};
  // owned copies of the inputs
  std::vector<double> q, sigma, x, beta, gamma;
  std::vector<int> species;
  double origin[3], cell[9];
  int periodic[3];
  size_t bytes = 0;
  // results
  btam_job_result res{};
  std::vector<double> q_out, sigma_out, x_out;
  bool done = false;
};

double since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

}  // namespace

// ---- the evaluation batcher -------------------------------------------------
// Launch variants of served evaluations (index 0 FP64, 1 FP32C): undirected,
// persistent grid, and the block shapes the autotuner picks for the plain
// drop-in workload on a B200.
constexpr int kServeVariant1[2] = {btam::kUndirected | btam::kPersistent | 3,
                                   btam::kUndirected | btam::kPersistent | 4};
constexpr int kServeVariant2[2] = {btam::kUndirected | btam::kPersistent | 0,
                                   btam::kUndirected | btam::kPersistent | 2};
// How long a round waits for the running jobs that have not asked yet.
constexpr int kRoundWaitUs = 400;
// Jobs of at most this many sites share the batched evaluations; larger
// jobs fill the GPU on their own and run their own kernels on their own
// streams (their launch and synchronisation overheads are a small part of
// their evaluations, and a shared round would make the small jobs wait for
// them).
constexpr int kBatchMaxSites = 8192;

struct EvalBatcher {
  int device = 0;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  struct Req {
    btam_system *s;
    int precision;
    bool done = false;
    int status = BTAM_OK;
  };
  std::vector<btam_system *> members;  // systems of the running jobs
  bool joined = false;                 // a member is missing from the batch layout
  std::vector<Req *> pending;
  Clock::time_point first_pending;
  // a round is running on a copy of the members: a job must not leave (and
  // destroy its system) until it ends
  bool in_round = false;
  // the batch and the systems of its layout (a system that left keeps its
  // rows until the next rebuild; they are evaluated but nobody reads them)
  btam_batch *batch = nullptr;
  std::map<btam_system *, int> layout;
  long long layout_sites = 0, departed_sites = 0;  // real sites in the layout; of jobs gone
  std::thread thr;
  long long rounds = 0, evals = 0, rebuilds = 0;
};

namespace {

// Builds the batch over the current members, with the served launch shapes.
int batcher_rebuild(EvalBatcher *B, const std::vector<btam_system *> &members) {
  if (B->batch) btam_batch_destroy(B->batch);
  B->batch = nullptr;
  B->layout.clear();
  if (members.empty()) return BTAM_OK;
  int st = btam_batch_create(members.data(), (int)members.size(), &B->batch);
  for (int f = 0; f < 2 && st == BTAM_OK; ++f)
    st = btam_batch_set_variants(B->batch, f == 0 ? BTAM_FP64 : BTAM_FP32C, kServeVariant1[f],
                                 kServeVariant2[f]);
  if (st != BTAM_OK) return st;
  B->layout_sites = 0;
  for (size_t k = 0; k < members.size(); ++k) {
    B->layout[members[k]] = (int)k;
    B->layout_sites += members[k]->n_real;
  }
  ++B->rebuilds;
  return BTAM_OK;
}

// One round: the requests of each precision in tables of at most
// BatchXfer::kMax systems, each table one gather, one batch evaluation and
// one scatter on the batch's stream; then every requester's done event.
int batcher_round(EvalBatcher *B, const std::vector<EvalBatcher::Req *> &round,
                  const std::vector<btam_system *> &members, bool rebuild) {
  if (rebuild) {
    int st = batcher_rebuild(B, members);
    if (st != BTAM_OK) return st;
  }
  for (int prec : {BTAM_FP32C, BTAM_FP64}) {
    std::vector<btam_system *> sys;
    for (auto *r : round)
      if (r->precision == prec) sys.push_back(r->s);
    for (size_t at = 0; at < sys.size(); at += BatchXfer::kMax) {
      BatchXfer t;
      cudaEvent_t ready[BatchXfer::kMax];
      const size_t end = std::min(sys.size(), at + BatchXfer::kMax);
      for (size_t j = at; j < end; ++j) {
        btam_system *s = sys[j];
        auto it = B->layout.find(s);
        if (it == B->layout.end()) return BTAM_ERR_ARG;  // not in the batch: cannot happen
        BatchXfer::Sys &d = t.sys[t.n];
        d.pos = s->pos;
        d.xb = s->xb;
        d.rho = s->rho;
        d.V0 = s->V0;
        d.S0 = s->S0;
        d.Rq = s->Rq;
        d.Rs = s->Rs;
        d.Rx = s->Rx;
        d.totals = s->totals;
        d.err = s->err;
        d.n = s->n_real;
        d.g = s->n_ghost;
        d.k = it->second;
        batch_bases(B->batch, d.k, &d.R, &d.G);
        ready[t.n] = s->batch_ready;
        ++t.n;
      }
      int st = batch_round(B->batch, t, ready, prec);
      if (st != BTAM_OK) return st;
      for (int j = 0; j < t.n; ++j)
        BTAM_TRY(cudaEventRecord(sys[at + j]->batch_done, batch_stream_of(B->batch)));
      B->evals += t.n;
    }
  }
  ++B->rounds;
  return BTAM_OK;
}

void batcher_main(EvalBatcher *B) {
  cudaSetDevice(B->device);
  std::unique_lock<std::mutex> lock(B->mu);
  for (;;) {
    // a round starts when every running job has asked, or when the first
    // request has waited kRoundWaitUs
    for (;;) {
      if (B->pending.empty()) {
        if (B->stop) break;
        B->cv.wait(lock);
        continue;
      }
      if (B->pending.size() >= B->members.size() || B->stop) break;
      const auto deadline = B->first_pending + std::chrono::microseconds(kRoundWaitUs);
      if (B->cv.wait_until(lock, deadline) == std::cv_status::timeout) break;
    }
    if (B->pending.empty()) return;  // stopping
    std::vector<EvalBatcher::Req *> round;
    round.swap(B->pending);
    const std::vector<btam_system *> members = B->members;
    // rebuild when a job joined, or when the rows of jobs that left are more
    // than a quarter of the batch (they are evaluated for nothing)
    bool rebuild = B->joined || !B->batch || 4 * B->departed_sites > B->layout_sites;
    for (auto *r : round)
      if (!B->layout.count(r->s)) rebuild = true;
    B->joined = false;
    if (rebuild) B->departed_sites = 0;
    B->in_round = true;
    lock.unlock();
    const int st = batcher_round(B, round, members, rebuild);
    lock.lock();
    B->in_round = false;
    for (auto *r : round) {
      r->status = st;
      r->done = true;
    }
    B->cv.notify_all();
  }
}

// Attaches a built system to the batcher (its evaluations then go there).
int batcher_attach(EvalBatcher *B, btam_system *s) {
  BTAM_TRY(cudaEventCreateWithFlags(&s->batch_ready, cudaEventDisableTiming));
  BTAM_TRY(cudaEventCreateWithFlags(&s->batch_done, cudaEventDisableTiming));
  std::lock_guard<std::mutex> lock(B->mu);
  B->members.push_back(s);
  B->joined = true;
  s->batcher = B;
  return BTAM_OK;
}

// Detaches a system whose work has finished (its stream is idle, so no round
// still reads or writes its buffers), once no round is running: a round
// works on a copy of the members and may be rebuilding the batch from it.
void batcher_detach(EvalBatcher *B, btam_system *s) {
  {
    std::unique_lock<std::mutex> lock(B->mu);
    // a running round may be rebuilding the batch from this system
    B->cv.wait(lock, [&] { return !B->in_round; });
    B->members.erase(std::find(B->members.begin(), B->members.end(), s));
    // its rows stay in the batch until the next rebuild
    if (B->layout.erase(s)) B->departed_sites += s->n_real;
    s->batcher = nullptr;
  }
  B->cv.notify_all();  // a round may have been waiting for this job
  if (s->batch_ready) cudaEventDestroy(s->batch_ready);
  if (s->batch_done) cudaEventDestroy(s->batch_done);
  s->batch_ready = s->batch_done = nullptr;
}

}  // namespace

// The served job's side: its state is ready once everything enqueued on its
// stream has run; the evaluation joins the next round, and the job's stream
// waits for that round's results.
int batcher_eval(btam_system *s, int precision) {
  EvalBatcher *B = s->batcher;
  BTAM_TRY(cudaEventRecord(s->batch_ready, s->st));
  EvalBatcher::Req r{s, precision};
  {
    std::unique_lock<std::mutex> lock(B->mu);
    if (B->pending.empty()) B->first_pending = Clock::now();
    B->pending.push_back(&r);
    B->cv.notify_all();
    B->cv.wait(lock, [&] { return r.done; });
  }
  if (r.status != BTAM_OK) return r.status;
  return cuda_status(cudaStreamWaitEvent(s->st, s->batch_done, 0));
}

struct btam_server {
  const btam_tables *T = nullptr;
  int device = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  btam::AdmissionQueue queue{0};
  std::map<long long, std::unique_ptr<Job>> jobs;
  long long next_id = 1;
  int running = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  long long completed = 0, failed = 0;
  EvalBatcher batcher;
};

namespace {

// Runs one job on the calling worker thread; fills job->res and the outputs.
void run_job(btam_server *srv, Job *job) {
  const btam_job_spec &sp = job->spec;
  btam_job_result &r = job->res;
  const int n = sp.n;
  btam_system *s = nullptr;
  int st = btam_system_create(srv->T, n, job->q.data(), job->sigma.data(), job->x.data(),
                              job->species.data(), job->beta.empty() ? nullptr : job->beta.data(),
                              job->gamma.empty() ? nullptr : job->gamma.data(), job->origin,
                              job->cell, job->periodic, &s);
  if (st == BTAM_OK) st = btam_neighbors_build(s, 0);
  // small jobs hand their evaluations to the batcher (the undirected
  // kernels on persistent grids, in the batch's buffers, which
  // btam_estimate_bytes counts); large jobs run the same kernels on their
  // own stream; a job that asks for the plain two-pass pair runs it alone
  bool attached = false;
  if (st == BTAM_OK && !sp.plain && n <= kBatchMaxSites) {
    st = batcher_attach(&srv->batcher, s);
    attached = st == BTAM_OK;
  } else if (st == BTAM_OK && !sp.plain) {
    st = btam_set_variants(s, BTAM_FP32C, kServeVariant1[1], kServeVariant2[1]);
    if (st == BTAM_OK) st = btam_set_variants(s, BTAM_FP64, kServeVariant1[0], kServeVariant2[0]);
  }
  if (st == BTAM_OK) {
    r.t_start = since(srv->t0);
    if (sp.kind == BTAM_JOB_RELAX) {
      double info[5] = {0, 0, 0, 0, 0};
      const double bounds[3] = {sp.sigma_min > 0 ? sp.sigma_min : 0.001,
                                sp.sigma_max > 0 ? sp.sigma_max : 0.4,
                                sp.x_min > 0 ? sp.x_min : 0.01};
      const int hist = sp.lbfgs_m > 0 ? sp.lbfgs_m : (sp.mode == BTAM_RELAX_NGMRES ? 3 : 8);
      st = btam_relax(s, sp.mode, sp.tol, sp.max_iter, hist, bounds, info);
      r.norm = info[0];
      r.iterations = (int)info[1];
      r.evaluations = (int)info[2];
      r.objective = info[3];
      r.converged = (int)info[4];
    } else if (sp.kind == BTAM_JOB_DMD) {
      st = btam_dmd_setup(s);
      long long tot[2] = {0, 0};
      if (st == BTAM_OK) st = btam_dmd_step(s, sp.precision, sp.nsteps, sp.dmd_params, tot);
      r.h_quanta_hi = tot[0];
      r.h_quanta_lo = tot[1];
      r.iterations = sp.nsteps;
    } else if (sp.kind == BTAM_JOB_STRETCH) {
      double F[3] = {1.0, 1.0, 1.0}, info[5] = {0, 0, 0, 0, 0};
      st = btam_relax_stretch(s, sp.tol > 0 ? sp.tol : 1e-12, 1e-10,
                              sp.max_iter > 0 ? sp.max_iter : 20, F, info);
      r.norm = info[0];
      r.iterations = (int)info[1];
      r.evaluations = (int)info[2];
      r.converged = info[3] > 0 ? 1 : 0;
      r.objective = F[0] * F[1] * F[2];
    } else if (sp.kind == BTAM_JOB_EVAL) {
      double totals[4] = {0, 0, 0, 0};
      st = btam_mf_eval(s, sp.precision, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                        totals);
      r.objective = totals[0];
      r.norm = totals[2];
      r.evaluations = 1;
    } else {
      st = BTAM_ERR_ARG;
    }
  }
  if (st == BTAM_OK) {
    job->q_out.resize(3 * (size_t)n);
    job->sigma_out.resize(n);
    job->x_out.resize(n);
    st = btam_system_get_state(s, job->q_out.data(), job->sigma_out.data(), job->x_out.data());
  }
  if (s) cudaStreamSynchronize(s->st);
  if (attached) batcher_detach(&srv->batcher, s);
  if (s) btam_system_destroy(s);
  r.status = st;
}

void worker_main(btam_server *srv) {
  cudaSetDevice(srv->device);
  std::unique_lock<std::mutex> lock(srv->mu);
  for (;;) {
    long long id = -1;
    srv->work_cv.wait(lock, [&] {
      if (srv->stop) return true;
      id = srv->queue.admit();
      return id >= 0;
    });
    if (id < 0) return;  // stopping
    Job *job = srv->jobs[id].get();
    job->res.t_admit = since(srv->t0);
    ++srv->running;
    lock.unlock();
    run_job(srv, job);
    lock.lock();
    job->res.t_end = since(srv->t0);
    job->done = true;
    --srv->running;
    srv->queue.release(job->bytes);
    if (job->res.status == BTAM_OK) ++srv->completed;
    else ++srv->failed;
    srv->done_cv.notify_all();
    srv->work_cv.notify_all();  // freed memory may admit waiting jobs
  }
}

}  // namespace

extern "C" {

long long btam_estimate_bytes(int n, const double cell[9], const int periodic[3]) {
  if (n <= 0) return 0;
  // images: each periodic direction adds a slab of width rc on both faces
  double grow = 1.0;
  for (int k = 0; k < 3; ++k) {
    if (!periodic || !periodic[k] || !cell) continue;
    const double *a = cell + 3 * ((k + 1) % 3), *b = cell + 3 * ((k + 2) % 3);
    const double *c = cell + 3 * k;
    double nx = a[1] * b[2] - a[2] * b[1], ny = a[2] * b[0] - a[0] * b[2],
           nz = a[0] * b[1] - a[1] * b[0];
    double area = std::sqrt(nx * nx + ny * ny + nz * nz);
    double vol = std::fabs(c[0] * nx + c[1] * ny + c[2] * nz);
    double h = area > 0 ? vol / area : 0.0;  // height of the cell along k
    grow *= h > 0 ? 1.0 + 2.0 * BTAM_R_CUTOFF / h : 3.0;
  }
  const double n_all = n * grow;
  // per all-sites row: position, occupancy/beta, species, owner, cell index,
  // cell slot, image code; per real site: state, staging, results, both
  // moment records, neighbour counts, the neighbour candidate buffer, the
  // neighbour list at the cap, master-equation state and graph, relaxation
  // vectors, and the undirected kernels' buffers at the cap (per slot:
  // reverse slot, owned-pair link and an FP64 slot record; per owned pair,
  // at most one per two slots: the pair and site indices and an FP64
  // pair-rule record); plus a fixed allowance for cells and library scratch
  const double per_all = 32 + 16 + 4 + 4 + 4 + 4 + 4;
  const double per_slot = 4 + 4 + 8 * 8 + 0.5 * (4 + 4 + (btam::kPrRec + 8) * 8);
  const double per_real = 8 + 40 + 48 + 24 + btam::kMomStride * 8 + btam::kMomStride * 4 + 8 + 256 * 4 +
                          BTAM_MAXNEIGH * 4 + 16 + 16 + 4 + BTAM_MAX_CHEMICAL_NEIGHS * 4 +
                          (2 * 8 + 8) * 5 * 8 + BTAM_MAXNEIGH * per_slot;
  return (long long)(n_all * per_all + n * per_real) + (8ll << 20);
}

int btam_server_create(const btam_tables *t, int n_workers, long long budget_bytes,
                       btam_server **out) {
  if (!t || !out || n_workers <= 0) return BTAM_ERR_ARG;
  *out = nullptr;
  btam_server *srv = new btam_server;
  srv->T = t;
  srv->t0 = Clock::now();
  if (cudaGetDevice(&srv->device) != cudaSuccess) {
    delete srv;
    return BTAM_ERR_CUDA;
  }
  if (budget_bytes <= 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      delete srv;
      return BTAM_ERR_CUDA;
    }
    budget_bytes = (long long)(0.8 * (double)free_b);
  }
  srv->queue = btam::AdmissionQueue((size_t)budget_bytes);
  srv->batcher.device = srv->device;
  srv->batcher.thr = std::thread(batcher_main, &srv->batcher);
  for (int w = 0; w < n_workers; ++w) srv->workers.emplace_back(worker_main, srv);
  *out = srv;
  return BTAM_OK;
}

int btam_server_submit(btam_server *srv, const btam_job_spec *sp, long long *job_id) {
  if (!srv || !sp || !job_id || sp->n <= 0 || !sp->q || !sp->sigma || !sp->x || !sp->species ||
      !sp->origin || !sp->cell || !sp->periodic)
    return BTAM_ERR_ARG;
  if (sp->kind != BTAM_JOB_RELAX && sp->kind != BTAM_JOB_DMD && sp->kind != BTAM_JOB_EVAL &&
      sp->kind != BTAM_JOB_STRETCH)
    return BTAM_ERR_ARG;
  auto job = std::make_unique<Job>();
  const size_t n = sp->n;
  job->spec = *sp;
  job->q.assign(sp->q, sp->q + 3 * n);
  job->sigma.assign(sp->sigma, sp->sigma + n);
  job->x.assign(sp->x, sp->x + n);
  job->species.assign(sp->species, sp->species + n);
  if (sp->beta) job->beta.assign(sp->beta, sp->beta + n);
  if (sp->gamma) job->gamma.assign(sp->gamma, sp->gamma + n);
  std::memcpy(job->origin, sp->origin, sizeof(job->origin));
  std::memcpy(job->cell, sp->cell, sizeof(job->cell));
  std::memcpy(job->periodic, sp->periodic, sizeof(job->periodic));
  // the spec keeps no caller pointers
  job->spec.q = job->spec.sigma = job->spec.x = job->spec.beta = job->spec.gamma = nullptr;
  job->spec.species = nullptr;
  job->spec.origin = job->spec.cell = nullptr;
  job->spec.periodic = nullptr;
  job->bytes = (size_t)btam_estimate_bytes(sp->n, job->cell, job->periodic);
  std::lock_guard<std::mutex> lock(srv->mu);
  if (srv->stop) return BTAM_ERR_ARG;
  if (!srv->queue.fits_ever(job->bytes)) return BTAM_ERR_TOO_LARGE;
  job->id = srv->next_id++;
  job->res.t_submit = since(srv->t0);
  job->res.kind = sp->kind;
  *job_id = job->id;
  srv->queue.push(job->id, job->bytes);
  srv->jobs[job->id] = std::move(job);
  srv->work_cv.notify_one();
  return BTAM_OK;
}

int btam_server_wait(btam_server *srv, long long job_id, double timeout_s, btam_job_result *res,
                     double *q, double *sigma, double *x) {
  if (!srv) return BTAM_ERR_ARG;
  std::unique_lock<std::mutex> lock(srv->mu);
  auto it = srv->jobs.find(job_id);
  if (it == srv->jobs.end()) return BTAM_ERR_ARG;
  Job *job = it->second.get();
  auto ready = [&] { return job->done; };
  if (timeout_s < 0) {
    srv->done_cv.wait(lock, ready);
  } else if (!srv->done_cv.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
    return BTAM_ERR_TIMEOUT;
  }
  if (res) *res = job->res;
  const size_t n = job->spec.n;
  if (job->res.status == BTAM_OK) {
    if (q) std::memcpy(q, job->q_out.data(), 3 * n * sizeof(double));
    if (sigma) std::memcpy(sigma, job->sigma_out.data(), n * sizeof(double));
    if (x) std::memcpy(x, job->x_out.data(), n * sizeof(double));
  }
  int st = job->res.status;
  srv->jobs.erase(it);  // a result is collected once
  return st;
}

int btam_server_stats(btam_server *srv, long long *waiting, int *running, long long *completed,
                      long long *failed, long long *bytes_in_use) {
  if (!srv) return BTAM_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->mu);
  if (waiting) *waiting = (long long)srv->queue.waiting();
  if (running) *running = srv->running;
  if (completed) *completed = srv->completed;
  if (failed) *failed = srv->failed;
  if (bytes_in_use) *bytes_in_use = (long long)srv->queue.in_use();
  return BTAM_OK;
}

int btam_server_destroy(btam_server *srv) {
  if (!srv) return BTAM_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->stop = true;
  }
  srv->work_cv.notify_all();
  for (auto &w : srv->workers) w.join();
  {
    std::lock_guard<std::mutex> lock(srv->batcher.mu);
    srv->batcher.stop = true;
  }
  srv->batcher.cv.notify_all();
  srv->batcher.thr.join();
  if (srv->batcher.batch) btam_batch_destroy(srv->batcher.batch);
  delete srv;
  return BTAM_OK;
}

int btam_server_batch_stats(btam_server *srv, long long *rounds, long long *evaluations,
                            long long *rebuilds) {
  if (!srv) return BTAM_ERR_ARG;
  std::lock_guard<std::mutex> lock(srv->batcher.mu);
  if (rounds) *rounds = srv->batcher.rounds;
  if (evaluations) *evaluations = srv->batcher.evals;
  if (rebuilds) *rebuilds = srv->batcher.rebuilds;
  return BTAM_OK;
}

}  // extern "C"
