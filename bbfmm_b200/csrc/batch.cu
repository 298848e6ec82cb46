// Batched solves of many independent particle sets of uneven size, order and depth.
//
// The reference solves one particle set per call (bbfmm.c:15-87); this is new. Sets with
// the same (n, depth) form a group and are stacked into one solver: set k of a group owns
// the Morton cell indices [k 8^l, (k+1) 8^l) of every level and the leaves
// [k 8^maxlev, (k+1) 8^maxlev), so every pass of the group (P2M, M2M, projections, each
// level's M2L, L2L, L2P, P2P) is ONE launch over all its sets, and the M2L class grid of a
// level is simply 8 x nsets classes deep. Groups of the same n share one copy of the
// operators. The groups run on their own streams, forked from and joined back into the
// batch stream, and the whole batch solve is captured once into a CUDA graph and replayed.
//
// Particles: the caller's arrays hold all sets back to back (set s at offset
// sum_{t<s} counts[t]); every group's permutation indexes those arrays directly, so q is
// read and phi written in place, each group touching only its own sets' entries. The trees
// are sorted on the host (positions in host memory) or on the device (positions in device
// memory: one stable radix sort per group over (set slot, leaf) keys), with the same result.
#include <algorithm>
#include <cstdio>
#include <map>
#include <memory>
#include <vector>

#include "../../include/bbfmm_b200.h"
#include "solver.cuh"

#define TRY_(x)                        \
  do {                                 \
    int rc__ = (x);                    \
    if (rc__ != BBFMM_OK) return rc__; \
  } while (0)

template <typename T>
int bbfmm_weights(int n, T *Tkz, int *Ktable, T *Kweights, T *Cweights);
template <typename T>
int bbfmm_sort_particles(int N, const T *xyz, T L, int maxlev, int *perm, int *leaf_start);

namespace bbfmm {

template <typename T>
struct Batch {
  struct Group {
    int n = 0, maxlev = 0;
    std::vector<int> sets;
    std::unique_ptr<Solver<T>> solver;
    cudaEvent_t done = nullptr;
  };
  int mode = MODE_D, device = 0;
  double L = 1.0;
  int nsets = 0;
  int64_t ntotal = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<Group> groups;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *graph_q = nullptr;
  void *graph_phi = nullptr;
  size_t graph_nodes = 0;

  ~Batch() { release(); }

  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    graph_q = nullptr;
    graph_phi = nullptr;
    graph_nodes = 0;
  }

  void release() {
    drop_graph();
    // solvers that borrow operators go before the ones that own them
    for (auto &g : groups)
      if (g.solver && !g.solver->own_ops) {
        g.solver->release();
        g.solver.reset();
      }
    for (auto &g : groups) {
      if (g.solver) g.solver->release();
      g.solver.reset();
      if (g.done) cudaEventDestroy(g.done);
      g.done = nullptr;
    }
    groups.clear();
    if (fork) cudaEventDestroy(fork);
    fork = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }

  int create(int mode_, double L_, int device_, int lead, int lead_rows, int nsets_, const int *n_of,
             const int *maxlev_of, const int *counts, const T *xyz, const void *const *U_by_n,
             const void *const *E_by_n, int ops_fp32, bool xyz_on_device = false) {
    mode = mode_;
    L = L_;
    device = device_;
    nsets = nsets_;
    if (nsets < 1) return bbfmm_set_error(BBFMM_ERR_ARG, "a batch needs at least one set");
    std::vector<int64_t> off(nsets + 1, 0);
    for (int s = 0; s < nsets; ++s) {
      if (counts[s] < 0) return bbfmm_set_error(BBFMM_ERR_ARG, "negative set size");
      if (n_of[s] != 4 && n_of[s] != 8) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
      if (maxlev_of[s] < BBFMM_MINLEV || maxlev_of[s] > 10) return bbfmm_set_error(BBFMM_ERR_ARG, "bad depth");
      off[s + 1] = off[s] + counts[s];
    }
    if (off[nsets] > 0x7fffffff) return bbfmm_set_error(BBFMM_ERR_ARG, "more than 2^31 - 1 particles in a batch");
    ntotal = off[nsets];
    BBFMM_CUDA_OK(cudaSetDevice(device));
    BBFMM_CUDA_OK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    BBFMM_CUDA_OK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    // groups by (n, depth), in that order
    std::map<std::pair<int, int>, std::vector<int>> by;
    for (int s = 0; s < nsets; ++s) by[{n_of[s], maxlev_of[s]}].push_back(s);
    std::map<int, Solver<T> *> owner;  // first solver of each n owns the operators
    for (auto &kv : by) {
      groups.emplace_back();  // owned by the batch at once, so a failure below still frees it
      Group &g = groups.back();
      g.n = kv.first.first;
      g.maxlev = kv.first.second;
      g.sets = kv.second;
      g.solver.reset(new Solver<T>());
      Solver<T> &sv = *g.solver;
      TRY_(sv.init(g.n, g.maxlev, L, mode, lead, lead_rows, device, nullptr));
      auto it = owner.find(g.n);
      if (it == owner.end()) {
        const int nn = g.n, n3 = nn * nn * nn, r = n3 / 2;
        const int k = nn == 4 ? 0 : 1;
        if (!U_by_n[k] || !E_by_n[k]) return bbfmm_set_error(BBFMM_ERR_ARG, "missing operators for an order in use");
        std::vector<T> Tkz(nn * nn), Kw(n3), Cw(2 * nn * nn);
        std::vector<int> Kt(343);
        TRY_(bbfmm_weights<T>(nn, Tkz.data(), Kt.data(), Kw.data(), Cw.data()));
        TRY_(sv.set_tables(Tkz.data(), Cw.data(), Kw.data()));
        const size_t nu = (size_t)n3 * r, ne = (size_t)BBFMM_NUM_OFFSETS * r * r;
        std::vector<T> U(nu), E(ne);
        for (size_t i = 0; i < nu; ++i)
          U[i] = ops_fp32 ? (T)((const float *)U_by_n[k])[i] : (T)((const double *)U_by_n[k])[i];
        for (size_t i = 0; i < ne; ++i)
          E[i] = ops_fp32 ? (T)((const float *)E_by_n[k])[i] : (T)((const double *)E_by_n[k])[i];
        TRY_(sv.set_operators(U.data(), E.data()));
        owner[g.n] = &sv;
      } else {
        TRY_(sv.share_operators(*it->second));
      }
      if (xyz_on_device) {  // the group's trees in one device sort
        std::vector<int> offs(g.sets.size()), cnts(g.sets.size());
        for (size_t j = 0; j < g.sets.size(); ++j) {
          offs[j] = (int)off[g.sets[j]];
          cnts[j] = counts[g.sets[j]];
        }
        TRY_(sv.set_particles_sets_device((int)g.sets.size(), offs.data(), cnts.data(), (int)ntotal, xyz));
        BBFMM_CUDA_OK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
        continue;
      }
      // per set: leaf sort on the host, then one permutation / leaf table over the group
      const int64_t nl = pow8i(g.maxlev);
      int64_t Ng = 0;
      for (int s : g.sets) Ng += counts[s];
      std::vector<int> perm(Ng > 0 ? Ng : 1), ls(g.sets.size() * nl + 1);
      int64_t base = 0;
      for (size_t j = 0; j < g.sets.size(); ++j) {
        const int s = g.sets[j];
        std::vector<int> ps(counts[s] > 0 ? counts[s] : 1), lss(nl + 1);
        TRY_(bbfmm_sort_particles<T>(counts[s], xyz + 3 * off[s], (T)L, g.maxlev, ps.data(), lss.data()));
        for (int k = 0; k < counts[s]; ++k) perm[base + k] = (int)(off[s] + ps[k]);
        for (int64_t m = 0; m < nl; ++m) ls[j * nl + m] = (int)(base + lss[m]);
        base += counts[s];
      }
      ls[g.sets.size() * nl] = (int)base;
      TRY_(sv.set_particles_global((int)g.sets.size(), (int)Ng, perm.data(), ls.data(), (int)ntotal, xyz));
      BBFMM_CUDA_OK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    }
    return BBFMM_OK;
  }

  // Every group after the batch stream's prior work, the batch stream after every group.
  int run(const void *q, void *phi, int io_double) {
    BBFMM_CUDA_OK(cudaEventRecord(fork, stream));
    for (auto &g : groups) {
      BBFMM_CUDA_OK(cudaStreamWaitEvent(g.solver->stream, fork, 0));
      TRY_(g.solver->solve(q, phi, io_double));
      BBFMM_CUDA_OK(cudaEventRecord(g.done, g.solver->stream));
      BBFMM_CUDA_OK(cudaStreamWaitEvent(stream, g.done, 0));
    }
    return BBFMM_OK;
  }

  int solve(const void *q, void *phi, int use_graph) {
    const int io_double = sizeof(T) == 8;
    if (!use_graph) return run(q, phi, io_double);
    if (!exec || graph_q != q || graph_phi != phi) {
      drop_graph();
      // relaxed: the launchers set function attributes (not stream work) while capturing
      BBFMM_CUDA_OK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
      int rc = run(q, phi, io_double);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(stream, &g);
      if (rc != BBFMM_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "batch graph capture", __FILE__, __LINE__);
      graph = g;
      BBFMM_CUDA_OK(cudaGraphGetNodes(graph, nullptr, &graph_nodes));
      BBFMM_CUDA_OK(cudaGraphInstantiate(&exec, graph, 0));
      graph_q = q;
      graph_phi = phi;
    }
    BBFMM_CUDA_OK(cudaGraphLaunch(exec, stream));
    return BBFMM_OK;
  }

  // Target regions of every set at level depth_s - levels_up: active holds, set after set,
  // the 8^(depth_s - levels_up) mask bytes of each set (null clears); with first_m2l the local
  // expansions of each group start one level below its region level.
  int set_target_regions(int levels_up, const unsigned char *active, int first_m2l) {
    drop_graph();
    std::vector<int64_t> off(nsets + 1, 0);
    std::vector<int> depth(nsets, 0);
    for (auto &g : groups)
      for (int s : g.sets) depth[s] = g.maxlev;
    for (int s = 0; s < nsets; ++s) {
      const int R = depth[s] - levels_up;
      if (active && (R < BBFMM_MINLEV || levels_up < 0))
        return bbfmm_set_error(BBFMM_ERR_ARG, "region level below 2 for a set of the batch");
      off[s + 1] = off[s] + (active ? pow8i(R) : 0);
    }
    for (auto &g : groups) {
      Solver<T> &sv = *g.solver;
      const int R = g.maxlev - levels_up;
      if (!active) {
        TRY_(sv.set_target_region(-1, nullptr));
        TRY_(sv.set_m2l_first(BBFMM_MINLEV));
        continue;
      }
      std::vector<unsigned char> m;
      m.reserve(g.sets.size() * pow8i(R));
      for (int s : g.sets) m.insert(m.end(), active + off[s], active + off[s + 1]);
      TRY_(sv.set_target_region(R, m.data()));
      TRY_(sv.set_m2l_first(first_m2l ? R + 1 : BBFMM_MINLEV));
    }
    return BBFMM_OK;
  }

  // Degree of homogeneity of the kernel of every group (Solver::homogen).
  int set_kernel(int hg) {
    drop_graph();
    for (auto &g : groups) g.solver->homogen = hg;
    return BBFMM_OK;
  }

  int autotune(const void *q) {
    drop_graph();
    for (auto &g : groups) TRY_(g.solver->autotune(q, sizeof(T) == 8));
    return BBFMM_OK;
  }
};

}  // namespace bbfmm

// ------------------------------------------------------------------------ C-ABI
struct bbfmm_b200_batch {
  std::unique_ptr<bbfmm::Batch<double>> d;
  std::unique_ptr<bbfmm::Batch<float>> f;
};

extern "C" {

static int batch_create(const bbfmm_b200_config *cfg, int nsets, const int *n, const int *maxlev, const int *counts,
                        const void *xyz, const void *U4, const void *E4, const void *U8, const void *E8,
                        int operators_fp32, bool xyz_on_device, bbfmm_b200_batch **out) {
  if (!cfg || !out || !n || !maxlev || !counts || (nsets > 0 && !xyz))
    return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  *out = nullptr;
  const void *U[2] = {U4, U8}, *E[2] = {E4, E8};
  std::unique_ptr<bbfmm_b200_batch> b(new bbfmm_b200_batch());
  int rc;
  if (cfg->mode == BBFMM_B200_MODE_S) {
    b->f.reset(new bbfmm::Batch<float>());
    rc = b->f->create(cfg->mode, cfg->L, cfg->device, cfg->lead, cfg->lead_rows, nsets, n, maxlev, counts,
                      (const float *)xyz, U, E, operators_fp32, xyz_on_device);
  } else {
    b->d.reset(new bbfmm::Batch<double>());
    rc = b->d->create(cfg->mode, cfg->L, cfg->device, cfg->lead, cfg->lead_rows, nsets, n, maxlev, counts,
                      (const double *)xyz, U, E, operators_fp32, xyz_on_device);
  }
  if (rc != BBFMM_OK) return rc;
  *out = b.release();
  return BBFMM_OK;
}

int bbfmm_b200_batch_create(const bbfmm_b200_config *cfg, int nsets, const int *n, const int *maxlev,
                            const int *counts, const void *xyz, const void *U4, const void *E4, const void *U8,
                            const void *E8, int operators_fp32, bbfmm_b200_batch **out) {
  return batch_create(cfg, nsets, n, maxlev, counts, xyz, U4, E4, U8, E8, operators_fp32, false, out);
}

int bbfmm_b200_batch_create_device(const bbfmm_b200_config *cfg, int nsets, const int *n, const int *maxlev,
                                   const int *counts, const void *xyz_dev, const void *U4, const void *E4,
                                   const void *U8, const void *E8, int operators_fp32, bbfmm_b200_batch **out) {
  return batch_create(cfg, nsets, n, maxlev, counts, xyz_dev, U4, E4, U8, E8, operators_fp32, true, out);
}

int bbfmm_b200_batch_solve(bbfmm_b200_batch *b, const void *q_dev, void *phi_dev, int use_graph) {
  if (!b || (!q_dev && (b->d ? b->d->ntotal : b->f->ntotal) > 0) || (!phi_dev && (b->d ? b->d->ntotal : b->f->ntotal) > 0))
    return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return b->d ? b->d->solve(q_dev, phi_dev, use_graph) : b->f->solve(q_dev, phi_dev, use_graph);
}

int bbfmm_b200_batch_autotune(bbfmm_b200_batch *b, const void *q_dev) {
  if (!b || !q_dev) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return b->d ? b->d->autotune(q_dev) : b->f->autotune(q_dev);
}

int bbfmm_b200_batch_set_target_regions(bbfmm_b200_batch *b, int levels_up, const unsigned char *active,
                                        int first_m2l) {
  if (!b) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return b->d ? b->d->set_target_regions(levels_up, active, first_m2l)
              : b->f->set_target_regions(levels_up, active, first_m2l);
}

int bbfmm_b200_batch_set_kernel(bbfmm_b200_batch *b, int kernel) {
  if (!b) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const int hg = bbfmm::kernel_homogen(kernel);
  if (!hg) return bbfmm_set_error(BBFMM_ERR_ARG, "unknown kernel");
  return b->d ? b->d->set_kernel(hg) : b->f->set_kernel(hg);
}

int bbfmm_b200_batch_groups(const bbfmm_b200_batch *b) {
  if (!b) return -bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return (int)(b->d ? b->d->groups.size() : b->f->groups.size());
}

long long bbfmm_b200_batch_graph_nodes(const bbfmm_b200_batch *b) {
  if (!b) return -bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return (long long)(b->d ? b->d->graph_nodes : b->f->graph_nodes);
}

int bbfmm_b200_batch_group_info(const bbfmm_b200_batch *b, int g, int *info) {
  if (!b || !info) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const int ng = bbfmm_b200_batch_groups(b);
  if (g < 0 || g >= ng) return bbfmm_set_error(BBFMM_ERR_ARG, "group index out of range");
  auto fill = [&](auto &grp) {
    const auto &sv = *grp.solver;
    info[0] = grp.n;
    info[1] = grp.maxlev;
    info[2] = (int)grp.sets.size();
    info[3] = sv.N;
    info[4] = sv.tune.p2p_threads;
    for (int l = 0; l <= 10; ++l) {
      info[5 + l] = sv.tune.m2l_kind[l];
      info[16 + l] = sv.tune.m2l_groups[l];
    }
  };
  if (b->d) fill(b->d->groups[g]);
  else fill(b->f->groups[g]);
  return BBFMM_OK;
}

int bbfmm_b200_batch_group_stage_times(bbfmm_b200_batch *b, int g, const void *q_dev, void *phi_dev, float *ms,
                                       int count) {
  if (!b || !ms || !q_dev || !phi_dev) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const int ng = bbfmm_b200_batch_groups(b);
  if (g < 0 || g >= ng) return bbfmm_set_error(BBFMM_ERR_ARG, "group index out of range");
  auto run = [&](auto &batch) -> int {
    auto &sv = *batch.groups[g].solver;
    BBFMM_CUDA_OK(cudaDeviceSynchronize());
    sv.timing = true;
    int rc = sv.solve(q_dev, phi_dev, sizeof(sv.pos4[0]) == 8);
    sv.timing = false;
    if (rc != BBFMM_OK) return rc;
    BBFMM_CUDA_OK(cudaStreamSynchronize(sv.stream));
    for (int i = 0; i < count && i < bbfmm::ST_COUNT; ++i) ms[i] = sv.stage_ms[i];
    return BBFMM_OK;
  };
  return b->d ? run(*b->d) : run(*b->f);
}

void *bbfmm_b200_batch_stream(bbfmm_b200_batch *b) {
  if (!b) return nullptr;
  return b->d ? (void *)b->d->stream : (void *)b->f->stream;
}

void bbfmm_b200_batch_destroy(bbfmm_b200_batch *b) { delete b; }

}  // extern "C"
