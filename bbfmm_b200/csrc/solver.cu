// Device-resident FMM solve: orchestration of the pass kernels, the M2L kernels and the
// near field, plus the handle-based C-ABI (include/bbfmm_b200.h).
//
// One solve (anotherFMMCompute.c:3-40 order):
//   gather q -> P2M (maxlev) -> [U-projection, M2M] up to level 2      (upward)
//   per level 2..maxlev: M2L -> post projection (assign) -> L2L from the parent level
//   L2P (assign) -> P2P (add) -> scatter phi to the caller's particle order
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/bbfmm_b200.h"
#include "solver.cuh"

template <typename T>
int bbfmm_weights(int n, T *Tkz, int *Ktable, T *Kweights, T *Cweights);
template <typename T>
int bbfmm_sort_particles(int N, const T *xyz, T L, int maxlev, int *perm, int *leaf_start);

static thread_local std::string g_last_error;

int bbfmm_set_error(int code, const char *msg) {
  if (code != BBFMM_OK) g_last_error = msg ? msg : "error";
  return code;
}

int bbfmm_set_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return BBFMM_OK;
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error '%s' in %s (%s:%d)", cudaGetErrorString(e), what, file, line);
  g_last_error = buf;
  return BBFMM_ERR_CUDA;
}

namespace bbfmm {

template <typename T>
static int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) return BBFMM_OK;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e != cudaSuccess) {
    *p = nullptr;
    char buf[160];
    snprintf(buf, sizeof(buf), "device allocation of %zu bytes failed (%s)", sizeof(T) * count,
             cudaGetErrorString(e));
    return bbfmm_set_error(BBFMM_ERR_NOMEM, buf);
  }
  return BBFMM_OK;
}

#define TRY(x)                       \
  do {                               \
    int rc__ = (x);                  \
    if (rc__ != BBFMM_OK) return rc__; \
  } while (0)

template <typename T>
Tables Solver<T>::tables() const {
  Tables t{};
  if (sizeof(T) == 8) {
    t.tkz_d = (const double *)tkz; t.cw_d = (const double *)cw; t.kw_d = (const double *)kw;
  } else {
    t.tkz_f = (const float *)tkz; t.cw_f = (const float *)cw; t.kw_f = (const float *)kw;
  }
  return t;
}

template <typename T>
int Solver<T>::init(int n_, int maxlev_, double L_, int mode_, int lead_, int lead_rows_, int device_, cudaStream_t s) {
  if (n_ != 4 && n_ != 8) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  if (maxlev_ < BBFMM_MINLEV || maxlev_ > 10) return bbfmm_set_error(BBFMM_ERR_ARG, "maxlev must be in [2, 10]");
  if (!(L_ > 0)) return bbfmm_set_error(BBFMM_ERR_ARG, "root length L must be positive");
  if (mode_ < MODE_D || mode_ > MODE_MIXED) return bbfmm_set_error(BBFMM_ERR_ARG, "unknown precision mode");
  if ((mode_ == MODE_S) != (sizeof(T) == 4)) return bbfmm_set_error(BBFMM_ERR_ARG, "precision mode / type mismatch");
  n = n_; n3 = n * n * n; r = n3 / 2; maxlev = maxlev_; L = L_; mode = mode_; device = device_;
  lead = (mode == MODE_MIXED) ? lead_ : 0;
  lead_rows = lead_rows_ > 0 ? lead_rows_ : r;
  if (mode == MODE_MIXED && (lead < 0 || lead > 64 || lead % 16 != 0))
    return bbfmm_set_error(BBFMM_ERR_ARG, "lead must be 0, 16, 32, 48 or 64");
  if (mode == MODE_MIXED && (lead_rows < 32 || lead_rows > r || lead_rows % 32 != 0))
    return bbfmm_set_error(BBFMM_ERR_ARG, "lead_rows must be a multiple of 32 in [32, r]");
  BBFMM_CUDA_OK(cudaSetDevice(device));
  if (s) {
    stream = s;
  } else {
    BBFMM_CUDA_OK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  std::vector<int> ot(8 * 189 * 4);
  build_offset_table(ot.data());
  TRY(dalloc(&offs, 8 * 189));
  BBFMM_CUDA_OK(cudaMemcpy(offs, ot.data(), sizeof(int) * ot.size(), cudaMemcpyHostToDevice));
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::set_tables(const T *Tkz_h, const T *Cw_h, const T *Kw_h) {
  if (!tkz) {
    TRY(dalloc(&tkz, n * n));
    TRY(dalloc(&cw, 2 * n * n));
    TRY(dalloc(&kw, n3));
  }
  BBFMM_CUDA_OK(cudaMemcpy(tkz, Tkz_h, sizeof(T) * n * n, cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaMemcpy(cw, Cw_h, sizeof(T) * 2 * n * n, cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaMemcpy(kw, Kw_h, sizeof(T) * n3, cudaMemcpyHostToDevice));
  // pageable copies may still be in flight when cudaMemcpy returns; the solver's stream does
  // not order after the legacy stream
  BBFMM_CUDA_OK(cudaDeviceSynchronize());
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::set_operators(const T *U, const T *E) {
  // either half may be omitted: U feeds the projections, E the M2L
  if (!kw) return bbfmm_set_error(BBFMM_ERR_STATE, "tables must be set before operators");
  if (U) {
    std::vector<T> kwh(n3);
    BBFMM_CUDA_OK(cudaMemcpy(kwh.data(), kw, sizeof(T) * n3, cudaMemcpyDeviceToHost));
    std::vector<T> bup((size_t)n3 * r), bdn((size_t)r * n3);
    for (int l = 0; l < n3; ++l)
      for (int i = 0; i < r; ++i) {
        bup[(size_t)l * r + i] = kwh[l] * U[(size_t)i * n3 + l];
        bdn[(size_t)i * n3 + l] = U[(size_t)i * n3 + l];
      }
    if (!Bup) {
      TRY(dalloc(&Bup, bup.size()));
      TRY(dalloc(&Bdn, bdn.size()));
    }
    BBFMM_CUDA_OK(cudaMemcpy(Bup, bup.data(), sizeof(T) * bup.size(), cudaMemcpyHostToDevice));
    BBFMM_CUDA_OK(cudaMemcpy(Bdn, bdn.data(), sizeof(T) * bdn.size(), cudaMemcpyHostToDevice));
    BBFMM_CUDA_OK(cudaDeviceSynchronize());
    if (mode == MODE_MIXED && r == 256 && sizeof(T) == 8) {
      std::vector<T> blead((size_t)n3 * PROJ_LEAD);
      for (int l = 0; l < n3; ++l)
        for (int i = 0; i < PROJ_LEAD; ++i) blead[(size_t)l * PROJ_LEAD + i] = bup[(size_t)l * r + i];
      if (!Bup_lead) TRY(dalloc(&Bup_lead, blead.size()));
      BBFMM_CUDA_OK(cudaMemcpy(Bup_lead, blead.data(), sizeof(T) * blead.size(), cudaMemcpyHostToDevice));
      if (tcproj) tc_free_projections(tcproj);
      tcproj = nullptr;
      TRY(tc_prepare_projections(n3, r, (const double *)Bup, (const double *)Bdn, PROJ_LEAD, &tcproj, stream));
      BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
    }
  }
  if (!E) return BBFMM_OK;
  std::vector<T> ert((size_t)BBFMM_NUM_OFFSETS * r * r);
  for (int k = 0; k < BBFMM_NUM_OFFSETS; ++k)
    for (int i = 0; i < r; ++i)
      for (int j = 0; j < r; ++j)
        ert[((size_t)k * r + i) * r + j] = E[((size_t)k * r + j) * r + i];
  if (!Ert) {
    TRY(dalloc(&Ert, ert.size()));
    TRY(dalloc(&Ecol, ert.size()));
  }
  BBFMM_CUDA_OK(cudaMemcpy(Ert, ert.data(), sizeof(T) * ert.size(), cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaMemcpy(Ecol, E, sizeof(T) * ert.size(), cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaDeviceSynchronize());
  if (mode == MODE_MIXED && r == 256) {  // r = 32 (n = 4): the M2L stays in FP64 on CUDA cores
    if (!tc_supported()) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "mixed mode needs an sm_100 GPU");
    if (tcops) tc_free_operators(tcops);
    tcops = nullptr;
    TRY(tc_prepare_operators(r, (const double *)Ert, lead, lead_rows, &tcops, stream));
    BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::share_operators(const Solver<T> &o) {
  if (o.n != n || o.mode != mode || o.lead != lead || o.lead_rows != lead_rows || o.device != device)
    return bbfmm_set_error(BBFMM_ERR_ARG, "operators can only be shared between solvers of the same n and mode");
  if (!o.Ert || !o.kw) return bbfmm_set_error(BBFMM_ERR_STATE, "the sharing solver has no operators");
  if (own_ops) {
    void *mine[] = {tkz, cw, kw, Ert, Ecol, Bup, Bdn, kwcol, Bup_lead};
    for (void *p : mine)
      if (p) cudaFree(p);
    if (tcops) tc_free_operators(tcops);
    if (tcproj) tc_free_projections(tcproj);
  }
  tkz = o.tkz; cw = o.cw; kw = o.kw; Ert = o.Ert; Ecol = o.Ecol; Bup = o.Bup; Bdn = o.Bdn; kwcol = o.kwcol;
  tcops = o.tcops;
  tcproj = o.tcproj;
  Bup_lead = o.Bup_lead;
  own_ops = false;
  return BBFMM_OK;
}

// Partial-sum scratch of the offset-group FP64 M2L for the current tuning.
template <typename T>
int Solver<T>::alloc_partials() {
  int64_t need = 0;
  {  // every full M2L (FP64 DMMA or SIMT) may split its offsets
    for (int l = BBFMM_MINLEV; l <= maxlev; ++l) {
      const bool tc = tc_m2l(l);
      if (tc) continue;
      const int g = tune.m2l_groups[l] > 0 ? tune.m2l_groups[l] : dmma_default_groups(l, nsets);
      const int64_t e = dmma_part_elems(l, nsets, g, r);
      if (e > need) need = e;
    }
  }
  if (need <= Lpart_elems && (need == 0 || Lpart)) return BBFMM_OK;
  if (Lpart) cudaFree(Lpart);
  Lpart = nullptr;
  Lpart_elems = 0;
  if (need > 0) {
    TRY(dalloc(&Lpart, (size_t)need));
    Lpart_elems = need;
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::alloc_work() {
  const int64_t nl = cells(maxlev);
  const int64_t cell_bytes = (int64_t)n3 * sizeof(T);
  if (slab_request > 0) slab = slab_request;
  else slab = nl * cell_bytes > ((int64_t)16 << 30) ? ((((int64_t)16 << 30) / cell_bytes) & ~(int64_t)63) : 0;
  int64_t smax[2] = {0, 0};
  for (int l = BBFMM_MINLEV; l <= maxlev; ++l) {
    const int64_t c = l == maxlev ? leaf_slab() : cells(l);
    if (c > smax[l & 1]) smax[l & 1] = c;
  }
  for (int b = 0; b < 2; ++b) {  // freed and cleared first: a failed allocation leaves no stale pointer
    if (S[b]) cudaFree(S[b]);
    if (F[b]) cudaFree(F[b]);
    S[b] = F[b] = nullptr;
    TRY(dalloc(&S[b], (size_t)smax[b] * n3));
    TRY(dalloc(&F[b], (size_t)smax[b] * n3));
  }
  Moff.assign(maxlev + 2, 0);
  int64_t tot = 0;
  for (int l = BBFMM_MINLEV; l <= maxlev; ++l) {
    Moff[l] = tot;
    tot += cells(l) * r;
  }
  if (Mall) cudaFree(Mall);
  TRY(dalloc(&Mall, (size_t)tot));
  // zeros where no pass writes (the cells outside a local solve's source region)
  BBFMM_CUDA_OK(cudaMemset(Mall, 0, sizeof(T) * (size_t)tot));
  if (Lbuf) cudaFree(Lbuf);
  TRY(dalloc(&Lbuf, (size_t)nl * r));
  TRY(alloc_partials());
  // bf16 copies of the projection inputs: the largest slab or level of S and of L rows
  if (Ssplit) cudaFree(Ssplit);
  if (Lsplit) cudaFree(Lsplit);
  Ssplit = Lsplit = nullptr;
  Ssplit_rows = Lsplit_rows = 0;
  if (proj_tc()) {
    int64_t sr = leaf_slab();
    for (int l = BBFMM_MINLEV; l < maxlev; ++l)
      if (cells(l) > sr) sr = cells(l);
    const int64_t lr = sr;  // both are used per slab of the leaf level and per whole level above
    unsigned char *p = nullptr;
    TRY(dalloc(&p, (size_t)sr * n3 * 4));
    Ssplit = p;
    Ssplit_rows = sr;
    if (lr > 0) {
      TRY(dalloc(&p, (size_t)lr * r * 4));
      Lsplit = p;
      Lsplit_rows = lr;
    }
  }
  if (mode == MODE_MIXED && r == 256) {
    if (Msplit) cudaFree(Msplit);
    Msplit = nullptr;
    unsigned char *p = nullptr;
    TRY(dalloc(&p, tc_split_bytes(r, tot / r)));
    Msplit = p;
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::set_particles_sorted(int N_, const int *perm_h, const int *leaf_start_h, const T *xyz_h) {
  return set_particles_global(1, N_, perm_h, leaf_start_h, N_, xyz_h);
}

template <typename T>
int Solver<T>::set_particles_global(int nsets_, int N_, const int *perm_h, const int *leaf_start_h, int Nxyz,
                                    const T *xyz_h) {
  if (nsets_ < 1 || nsets_ * pow8i(maxlev) > (int64_t)1 << 30)
    return bbfmm_set_error(BBFMM_ERR_ARG, "number of stacked sets out of range");
  nsets = nsets_;
  const int64_t nl = cells(maxlev);
  if (perm) { cudaFree(perm); cudaFree(leaf_start); cudaFree(pos4); cudaFree(phis); }
  if (near_work) cudaFree(near_work);
  near_work = nullptr;
  near_items = near_threads = 0;
  if (flds) cudaFree(flds);  // sized 3 N: reallocated by the next solve_fields
  for (T *p : {phis2, flds2, qs2, phisn, fldsn})
    if (p) cudaFree(p);
  phis2 = flds2 = qs2 = phisn = fldsn = nullptr;
  if (io_q) cudaFree(io_q);  // sized N: reallocated by the next host-buffer solve
  if (io_phi) cudaFree(io_phi);
  io_q = io_phi = nullptr;
  perm = leaf_start = nullptr; pos4 = phis = flds = nullptr;
  N = N_;
  TRY(dalloc(&perm, N > 0 ? N : 1));
  TRY(dalloc(&leaf_start, nl + 1));
  TRY(dalloc(&pos4, 4 * (size_t)(N > 0 ? N : 1)));
  TRY(dalloc(&phis, N > 0 ? N : 1));
  if (N > 0) BBFMM_CUDA_OK(cudaMemcpy(perm, perm_h, sizeof(int) * N, cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaMemcpy(leaf_start, leaf_start_h, sizeof(int) * (nl + 1), cudaMemcpyHostToDevice));
  BBFMM_CUDA_OK(cudaDeviceSynchronize());
  TRY(build_near_work());
  if (N > 0) {
    T *xyz_d = nullptr;
    TRY(dalloc(&xyz_d, 3 * (size_t)Nxyz));
    BBFMM_CUDA_OK(cudaMemcpyAsync(xyz_d, xyz_h, sizeof(T) * 3 * Nxyz, cudaMemcpyHostToDevice, stream));
    int rc = launch_gather<T, T>(N, perm, xyz_d, nullptr, pos4, stream);
    cudaStreamSynchronize(stream);
    cudaFree(xyz_d);
    TRY(rc);
  }
  TRY(alloc_work());
  BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
  return BBFMM_OK;
}

// The same state as set_particles_sorted for one set, with the octree built on the device from
// positions there (build_tree_device: the host sort's perm and leaf_start, bit for bit).
template <typename T>
int Solver<T>::set_particles_device(int N_, const T *xyz_d) {
  if (N_ < 0 || (N_ > 0 && !xyz_d)) return bbfmm_set_error(BBFMM_ERR_ARG, "bad particle arguments");
  const int off = 0;
  return set_particles_sets_device(1, &off, &N_, N_, xyz_d);
}

// The same state as set_particles_global, with the stacked sets' octrees built on the device
// (build_tree_device_sets: per set the host sort's perm and leaf_start, bit for bit).
template <typename T>
int Solver<T>::set_particles_sets_device(int nsets_, const int *off_h, const int *count_h, int Nxyz, const T *xyz_d) {
  if (nsets_ < 1 || nsets_ * pow8i(maxlev) > (int64_t)1 << 30)
    return bbfmm_set_error(BBFMM_ERR_ARG, "number of stacked sets out of range");
  int64_t total = 0;
  for (int j = 0; j < nsets_; ++j) {
    if (count_h[j] < 0 || off_h[j] < 0 || (int64_t)off_h[j] + count_h[j] > Nxyz)
      return bbfmm_set_error(BBFMM_ERR_ARG, "set range outside the positions array");
    total += count_h[j];
  }
  if (total > 0x7fffffff) return bbfmm_set_error(BBFMM_ERR_ARG, "more than 2^31 - 1 particles");
  if (total > 0 && !xyz_d) return bbfmm_set_error(BBFMM_ERR_ARG, "bad particle arguments");
  const int N_ = (int)total;
  nsets = nsets_;
  const int64_t nl = cells(maxlev);
  if (perm) { cudaFree(perm); cudaFree(leaf_start); cudaFree(pos4); cudaFree(phis); }
  if (near_work) cudaFree(near_work);
  near_work = nullptr;
  near_items = near_threads = 0;
  if (flds) cudaFree(flds);
  for (T *p : {phis2, flds2, qs2, phisn, fldsn})
    if (p) cudaFree(p);
  phis2 = flds2 = qs2 = phisn = fldsn = nullptr;
  if (io_q) cudaFree(io_q);
  if (io_phi) cudaFree(io_phi);
  io_q = io_phi = nullptr;
  perm = leaf_start = nullptr; pos4 = phis = flds = nullptr;
  N = N_;
  TRY(dalloc(&perm, N > 0 ? N : 1));
  TRY(dalloc(&leaf_start, nl + 1));
  TRY(dalloc(&pos4, 4 * (size_t)(N > 0 ? N : 1)));
  TRY(dalloc(&phis, N > 0 ? N : 1));
  TRY(build_tree_device_sets<T>(nsets, off_h, count_h, xyz_d, (T)L, maxlev, perm, leaf_start, stream));
  TRY(build_near_work());
  if (N > 0) TRY((launch_gather<T, T>(N, perm, xyz_d, nullptr, pos4, stream)));
  TRY(alloc_work());
  BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
  return BBFMM_OK;
}

template <typename T>
void Solver<T>::mark(int stage, int launches) {
  kernel_launches += launches;
  if (!timing) return;
  if (stage < 0) {
    cudaEventRecord(ev[ST_COUNT], stream);
    return;
  }
  // attribute the time since the previous mark to this stage
  static_assert(ST_COUNT + 1 <= (int)(sizeof(ev) / sizeof(ev[0])), "event table");
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, stream);
  cudaEventSynchronize(e);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, ev[ST_COUNT], e);
  stage_ms[stage] += ms;
  cudaEventDestroy(ev[ST_COUNT]);
  ev[ST_COUNT] = e;
}

template <typename T>
int Solver<T>::upward(const void *q_dev, int q_is_double) {
  const Tables tb = tables();
  if (q_dev) {
    if (q_is_double) TRY((launch_gather<T, double>(N, perm, nullptr, (const double *)q_dev, pos4, stream)));
    else TRY((launch_gather<T, float>(N, perm, nullptr, (const float *)q_dev, pos4, stream)));
    mark(ST_GATHER);
  }
  // leaf level, slab by slab (a local solve: its source runs): P2M, up projection, M2M into
  // the parents; the multipoles of the levels below m2l_first are not needed in a local solve
  // (a local solve: its source cells in compact order, and no level below m2l_first)
  const int lowest = local_solve ? m2l_first : BBFMM_MINLEV;
  auto count = [&](int l) { return local_solve ? n_src[l] : cells(l); };
  T *Sl = S[maxlev & 1];
  const int64_t *lr = local_solve ? src_list[maxlev] : nullptr;
  const int64_t nl = count(maxlev), sl = leaf_slab();
  for (int64_t a = 0; a < nl; a += sl) {
    const int64_t c = nl - a < sl ? nl - a : sl;
    // mixed mode: P2M also writes the BF16 split of S that the tensor-core up projection reads
    void *sp = proj_tc() && c <= Ssplit_rows ? Ssplit : nullptr;
    TRY(launch_p2m<T>(n, pos4, leaf_start, maxlev, (T)L, tb, Sl, stream, nsets, a, c, sp, lr ? lr + a : nullptr));
    mark(ST_P2M);
    TRY(proj_up(c, Sl, maxlev, a, sp != nullptr, lr ? lr + a : nullptr));
    mark(ST_PROJ_UP);
    if (maxlev - 1 >= lowest) {
      TRY(launch_m2m<T>(n, Sl, S[(maxlev - 1) & 1], maxlev - 1, tb, stream, nsets, a / 8, c / 8));
      mark(ST_M2M);
    }
  }
  for (int l = maxlev - 1; l >= lowest; --l) {
    if (l < maxlev - 1) {
      TRY(launch_m2m<T>(n, S[(l + 1) & 1], S[l & 1], l, tb, stream, nsets, 0, count(l)));
      mark(ST_M2M);
    }
    TRY(proj_up(count(l), S[l & 1], l, 0, false, local_solve ? src_list[l] : nullptr));
    mark(ST_PROJ_UP);
  }
  if (mode == MODE_MIXED && tcops) {
    TRY(tc_split_multipoles(r, Mcells(), (const double *)Mall, lead, Msplit, stream));
    mark(ST_PROJ_UP);
  }
  return BBFMM_OK;
}

// FP64 with r = 256 runs on the FP64 tensor path (DMMA); FP32 and r = 32 on CUDA cores.
template <typename T>
int Solver<T>::m2l_fp(const T *Ml, int level, int j0, int j1, int ni, const int4 *boxes, int nboxes) {
  if (sizeof(T) == 8 && r == 256)
    return launch_m2l_dmma(r, (const double *)Ml, (const double *)Ecol, (double *)Lbuf, level, j0, j1, ni, offs,
                           (double *)Lpart, Lpart_elems, stream, nsets, tune.m2l_groups[level], boxes, nboxes);
  // the SIMT kernel writes all r outputs; in the rank mode (ni = rk()) the outputs i >= rank
  // of the zero-padded operators come out as zeros, so only other partial ranges are refused
  if (ni != r && ni != rk())
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "partial output range needs the FP64 r = 256 path");
  const int g = tune.m2l_groups[level] > 0 ? tune.m2l_groups[level] : dmma_default_groups(level, nsets);
  return launch_m2l_simt<T>(r, Ml, Ert, Lbuf, level, j0, j1, offs, 0, stream, nsets, g, Lpart, Lpart_elems, boxes,
                            nboxes);
}

template <typename T>
int Solver<T>::proj(int64_t Mrows, int K, int Ncols, const T *A, const T *B, const T *cs, T scale, T *C, int level,
                    int mapmode, int64_t row0, int lda, const int64_t *rowlist) {
  if (sizeof(T) == 8) {
    int rc = launch_proj_dmma(Mrows, K, Ncols, (const double *)A, (const double *)B, (const double *)cs,
                              (double)scale, (double *)C, level, mapmode, stream, row0, lda, rowlist);
    if (rc != BBFMM_ERR_UNSUPPORTED) return rc;
  }
  return launch_proj<T>(Mrows, K, Ncols, A, nullptr, B, cs, scale, C, level, mapmode, stream, row0, 0, lda, rowlist);
}

// Up projection of `rows` S rows (Morton cells row0 .. of `level`) into the level's M (cpg).
// Mixed mode: components j < PROJ_LEAD in FP64, the rest as split-BF16 tensor-core products.
template <typename T>
int Solver<T>::proj_up(int64_t rows, const T *S_rows, int level, int64_t row0, bool presplit,
                       const int64_t *rowlist) {
  T *Mdst = Mall + Moff[level];
  if (!proj_tc() || rows > Ssplit_rows)
    return proj(rows, n3, r, S_rows, Bup, nullptr, (T)1, Mdst, level, MAP_OUT_CPG, row0, 0, rowlist);
  // the tensor cores write all r columns (zero for j < PROJ_LEAD: those operator rows are
  // zero in the split copy), then the FP64 pass overwrites the leading columns
  if (!presplit) TRY(tc_split_rows(rows, n3, (const double *)S_rows, 0, level, row0, Ssplit, stream));
  TRY(launch_proj_up(tcproj, Ssplit, rows, (double *)Mdst, level, row0, stream, rowlist));
  return launch_proj_narrow(rows, n3, (const double *)S_rows, (const double *)Bup_lead, (double *)Mdst, r, level,
                            MAP_OUT_CPG, stream, row0, rowlist);
}

// Down projection of the level's M2L output (Lbuf, cpg) into `rows` F rows (Morton cells
// row0 .., assign). Mixed mode: one pass, the contraction over j < 16 in FP64 and the rest on
// the tensor cores from L rows gathered into Morton order as split BF16.
template <typename T>
int Solver<T>::proj_down(int level, int64_t rows, int64_t row0, T *F_rows, bool presplit, const int64_t *rowlist) {
  // (1/L_l)^homogen in T, as the reference's POW(iL, homogen) (anotherFMMInteraction.c:7545-7549)
  const T iL = (T)1 / cell_length<T>(level, (T)L);
  const T scale = homogen == 1 ? iL : (T)std::pow(iL, (T)homogen);
  if (!proj_tc() || rows > Lsplit_rows)  // contraction over the effective rank (j < rk())
    return proj(rows, rk(), n3, Lbuf, Bdn, kw, scale, F_rows, level, MAP_IN_CPG, row0, r, rowlist);
  // components j < 16 in FP64 and the rest as split-BF16 tensor-core products, one pass
  if (!presplit) TRY(tc_split_rows(rows, r, (const double *)Lbuf, 1, level, row0, Lsplit, stream, 16, rowlist));
  return launch_proj_down(tcproj, Lsplit, (const double *)Lbuf, rows, (double *)F_rows, level, row0,
                          (const double *)kw, (double)scale, stream, rk(), rowlist);
}

// Leaf level after the M2L: per slab, the down projection of the M2L output (assign), L2L
// from the parents (add), then L2P (assign) -- the order of the whole-level path.
template <typename T>
int Solver<T>::leaf_down(bool field) {
  const Tables tb = tables();
  T *Fl = F[maxlev & 1];
  if (local_solve) {  // targets outside the region's leaf runs get zero
    BBFMM_CUDA_OK(cudaMemsetAsync(phis, 0, sizeof(T) * (size_t)(N > 0 ? N : 1), stream));
    if (field) BBFMM_CUDA_OK(cudaMemsetAsync(flds, 0, sizeof(T) * 3 * (size_t)(N > 0 ? N : 1), stream));
  }
  // slabs of the leaf level, or of a local solve's target leaves in compact order
  const int64_t *lr = local_solve ? tgt_list[maxlev] : nullptr;
  const int64_t nl = local_solve ? n_tgt[maxlev] : cells(maxlev), sl = leaf_slab();
  for (int64_t a = 0; a < nl; a += sl) {
    const int64_t c = nl - a < sl ? nl - a : sl;
    const int64_t *rl = lr ? lr + a : nullptr;
    if (chunked()) {
      TRY(proj_down(maxlev, c, a, Fl, false, rl));
      mark(ST_PROJ_DOWN);
      if (maxlev > m2l_first) {
        TRY(launch_l2l<T>(n, F[(maxlev - 1) & 1], Fl, maxlev - 1, tb, stream, nsets, a / 8, c / 8));
        mark(ST_L2L);
      }
    }
    if (field)
      TRY(launch_l2p_field<T>(n, pos4, leaf_start, maxlev, (T)L, tb, Fl, phis, flds, stream, nsets, a, c, rl));
    else TRY(launch_l2p<T>(n, pos4, leaf_start, maxlev, (T)L, tb, Fl, phis, stream, nsets, a, c, rl));
    mark(ST_L2P);
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::interaction(int lo, int hi) {
  const Tables tb = tables();
  for (int l = lo; l <= hi; ++l) {
    TRY(m2l_post(l));
    if (l > m2l_first && !(l == maxlev && chunked())) {  // chunked leaf level: in leaf_down
      TRY(launch_l2l<T>(n, F[(l - 1) & 1], F[l & 1], l - 1, tb, stream, nsets, 0,
                        local_solve ? n_tgt[l - 1] : cells(l - 1)));
      mark(ST_L2L);
    }
  }
  return BBFMM_OK;
}

// M2L of one level into Lbuf, then the post-M2L projection into F[l & 1] (assign).
template <typename T>
int Solver<T>::m2l_post(int l) {
  {
    const T *Ml = Mall + Moff[l];
    bool presplit = false;  // the M2L kernel wrote the split rows of the down projection
    const bool split = tc_m2l(l);
    if (split) {
      // FP64 leading block (i < lead_rows, j < lead) on the FP64 tensor path, then the
      // split-bf16 tensor-core kernel adds everything else into the same FP64 output; the
      // two-box kernel computes the block itself in its otherwise idle epilogue warps
      if (lead > 0 && tc_fuses_lead(tcops, tc_products, rk())) {
        // a target region: only the tiles above active cells run, the rest of the output is zero
        const bool masked = region_tcboxes[l] != nullptr;
        // whole level with mixed projections: the kernel also writes the split rows that the
        // down projection reads (and the FP64 output only where that pass reads it)
        presplit = !masked && proj_tc() && cells(l) <= Lsplit_rows && !(l == maxlev && chunked());
        if (masked) BBFMM_CUDA_OK(cudaMemsetAsync(Lbuf, 0, sizeof(T) * (size_t)cells(l) * r, stream));
        TRY(launch_m2l_tc(r, Msplit, Mcells(), Moff[l] / r, tcops, (double *)Lbuf, l, offs, stream, nsets,
                          tc_products, rk(), (const double *)Ml, (const double *)Ert, presplit ? Lsplit : nullptr,
                          region_tcboxes[l], region_ntcboxes[l], region_tcgeom[l]));
        mark(ST_M2L, 1);
      } else if (lead > 0) {
        TRY(m2l_fp(Ml, l, 0, lead, lead_rows));
        TRY(launch_m2l_tc(r, Msplit, Mcells(), Moff[l] / r, tcops, (double *)Lbuf, l, offs, stream, nsets,
                          tc_products, rk()));
        mark(ST_M2L, 2);
      } else {
        TRY(launch_m2l_tc(r, Msplit, Mcells(), Moff[l] / r, tcops, (double *)Lbuf, l, offs, stream, nsets,
                          tc_products, rk()));
        mark(ST_M2L, 1);
      }
    } else if (region_boxes[l]) {
      // a target region: only the blocks above active cells run (one offset group), the rest
      // of the output is zero
      BBFMM_CUDA_OK(cudaMemsetAsync(Lbuf, 0, sizeof(T) * (size_t)cells(l) * r, stream));
      TRY(m2l_fp(Ml, l, 0, rk(), rk(), region_boxes[l], region_nboxes[l]));
      mark(ST_M2L, 1);
    } else {
      TRY(m2l_fp(Ml, l, 0, rk(), rk()));
      int g = tune.m2l_groups[l] > 0 ? tune.m2l_groups[l] : dmma_default_groups(l, nsets);
      if ((int64_t)g * cells(l) * r > Lpart_elems) g = 1;
      mark(ST_M2L, g > 1 ? 2 : 1);  // groups add the partial sum
    }
    if (!(l == maxlev && chunked())) {  // chunked leaf level: in leaf_down
      TRY(proj_down(l, local_solve ? n_tgt[l] : cells(l), 0, F[l & 1], presplit, local_solve ? tgt_list[l] : nullptr));
      mark(ST_PROJ_DOWN);
    }
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::downward_finish(void *phi_dev, int phi_is_double, bool near) {
  const Tables tb = tables();
  TRY(leaf_down(false));
  if (near) TRY(this->near(phis, nullptr));
  if (phi_dev) {
    if (phi_is_double) TRY((launch_scatter<T, double>(N, perm, phis, (double *)phi_dev, stream)));
    else TRY((launch_scatter<T, float>(N, perm, phis, (float *)phi_dev, stream)));
    mark(ST_SCATTER);
  }
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::solve(const void *q_dev, void *phi_dev, int io_double) {
  if (!pos4) return bbfmm_set_error(BBFMM_ERR_STATE, "particles not set");
  if (!Ert) return bbfmm_set_error(BBFMM_ERR_STATE, "operators not set");
  kernel_launches = 0;
  if (timing) {
    for (int i = 0; i < ST_COUNT; ++i) stage_ms[i] = 0.f;
    if (!ev[ST_COUNT]) cudaEventCreate(&ev[ST_COUNT]);
    mark(-1, 0);
  }
  TRY(upward(q_dev, io_double));
  TRY(interaction(m2l_first, maxlev));
  TRY(downward_finish(phi_dev, io_double, true));
  return BBFMM_OK;
}

// Re-runs the M2L of one level `reps` times between two events on the solver's stream
// (multipoles of the last solve as input) and reports the mean time per launch group.
template <typename T>
int Solver<T>::time_m2l(int level, int reps, float *ms) {
  if (level < BBFMM_MINLEV || level > maxlev || reps < 1) return bbfmm_set_error(BBFMM_ERR_ARG, "bad level/reps");
  cudaEvent_t a, b;
  BBFMM_CUDA_OK(cudaEventCreate(&a));
  BBFMM_CUDA_OK(cudaEventCreate(&b));
  const T *Ml = Mall + Moff[level];
  const bool split = tc_m2l(level);
  const bool fused = split && lead > 0 && tc_fuses_lead(tcops, tc_products, rk());
  // the launch as the solve makes it: a whole level with the mixed projections also writes
  // the split rows of the down projection (m2l_post)
  const bool presplit = fused && proj_tc() && cells(level) <= Lsplit_rows && !(level == maxlev && chunked()) &&
                        !region_tcboxes[level];
  int rc = BBFMM_OK;
  float tot[2] = {0.f, 0.f};
  for (int part = 0; part < (split ? 2 : 1) && rc == BBFMM_OK; ++part) {
    cudaEventRecord(a, stream);
    for (int i = 0; i < reps && rc == BBFMM_OK; ++i) {
      if (!split) rc = m2l_fp(Ml, level, 0, rk(), rk());
      else if (part == 0) rc = launch_m2l_tc(r, Msplit, Mcells(), Moff[level] / r, tcops, (double *)Lbuf, level, offs,
                                             stream, nsets, tc_products, rk(), fused ? (const double *)Ml : nullptr,
                                             fused ? (const double *)Ert : nullptr, presplit ? Lsplit : nullptr);
      else rc = lead > 0 && !fused ? m2l_fp(Ml, level, 0, lead, lead_rows) : BBFMM_OK;
    }
    cudaEventRecord(b, stream);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&tot[part], a, b);
  }
  ms[0] = tot[0] / reps;
  ms[1] = tot[1] / reps;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

// Near field into the sorted potential (and field when fld != null), added.
template <typename T>
int Solver<T>::near(T *pot, T *fld) {
  if (near_threads != tune.p2p_threads) TRY(build_near_work());
  // The mixed mode's 1/r^4 near field runs in FP64: that kernel's potentials are near-field
  // dominated and its FP64 FMM error (3e-11 against the direct sum at n = 8) is far below the
  // ~1e-7 relative rounding of FP32 pair terms; its M2L and projections stay split-BF16.
  const int near_mode = mode == MODE_MIXED && homogen == 4 ? (int)MODE_D : mode;
  TRY(launch_near(near_mode, homogen, N, pos4, leaf_start, maxlev, near_work, nsets, near_items, near_threads, pot,
                  fld, stream, region_mask, region_level));
  mark(ST_P2P);
  return BBFMM_OK;
}

// Target region: active cells of `level` (8^level bytes, Morton order, host); level < 0 clears.
template <typename T>
int Solver<T>::set_target_region(int level, const unsigned char *active_host) {
  for (int l = 0; l <= 10; ++l) {
    if (region_boxes[l]) cudaFree(region_boxes[l]);
    if (region_tcboxes[l]) cudaFree(region_tcboxes[l]);
    region_boxes[l] = region_tcboxes[l] = nullptr;
    region_nboxes[l] = region_ntcboxes[l] = 0;
  }
  if (region_mask) cudaFree(region_mask);
  region_mask = nullptr;
  region_host.clear();
  region_level = -1;
  if (level >= 0) {
    if (level < BBFMM_MINLEV || level > maxlev || !active_host)
      return bbfmm_set_error(BBFMM_ERR_ARG, "target region: level in [2, maxlev] and a mask of nsets 8^level bytes");
    region_host.assign(active_host, active_host + cells(level));
    TRY(dalloc(&region_mask, (size_t)cells(level)));
    BBFMM_CUDA_OK(cudaMemcpy(region_mask, region_host.data(), region_host.size(), cudaMemcpyHostToDevice));
    region_level = level;
    TRY(build_region_tiles());
  }
  TRY(build_local());
  return pos4 ? build_near_work() : BBFMM_OK;
}

template <typename T>
int Solver<T>::set_m2l_first(int level) {
  if (level < BBFMM_MINLEV || level > maxlev) return bbfmm_set_error(BBFMM_ERR_ARG, "first M2L level in [2, maxlev]");
  m2l_first = level;
  return build_local();
}

template <typename T>
void Solver<T>::free_local() {
  for (int l = 0; l <= 10; ++l) {
    if (src_list[l]) cudaFree(src_list[l]);
    if (tgt_list[l]) cudaFree(tgt_list[l]);
    src_list[l] = tgt_list[l] = nullptr;
    n_src[l] = n_tgt[l] = 0;
  }
}

// Runs of the region cells (tgt) and of those with their neighbours (src) at region_level,
// then their cells at every level from m2l_first down to the leaves as device row lists.
template <typename T>
int Solver<T>::build_local() {
  free_local();
  src_runs.clear();
  tgt_runs.clear();
  local_solve = region_level >= BBFMM_MINLEV && m2l_first > region_level;
  if (!local_solve) return BBFMM_OK;
  const int R = region_level, m = 1 << R;
  const int64_t per = pow8i(R);
  std::vector<unsigned char> near((size_t)per);
  auto append = [](std::vector<std::pair<int64_t, int64_t>> &runs, int64_t row) {
    if (!runs.empty() && runs.back().first + runs.back().second == row) ++runs.back().second;
    else runs.push_back({row, 1});
  };
  for (int set = 0; set < nsets; ++set) {
    const unsigned char *act = region_host.data() + (size_t)set * per;
    std::fill(near.begin(), near.end(), (unsigned char)0);
    for (int64_t i = 0; i < per; ++i) {
      if (!act[i]) continue;
      int x, y, z;
      morton_to_grid(i, R, x, y, z);
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int u = x + dx, v = y + dy, w = z + dz;
            if (u >= 0 && u < m && v >= 0 && v < m && w >= 0 && w < m) near[(size_t)grid_to_morton(u, v, w, R)] = 1;
          }
    }
    for (int64_t i = 0; i < per; ++i) {
      if (near[(size_t)i]) append(src_runs, set * per + i);
      if (act[i]) append(tgt_runs, set * per + i);
    }
  }
  auto upload = [&](const std::vector<std::pair<int64_t, int64_t>> &runs, int l, int64_t **dst, int64_t *count) -> int {
    const int sh = 3 * (l - R);
    std::vector<int64_t> rows;
    for (const auto &ru : runs)
      for (int64_t c = ru.first << sh; c < (ru.first + ru.second) << sh; ++c) rows.push_back(c);
    *count = (int64_t)rows.size();
    TRY(dalloc(dst, rows.size() > 0 ? rows.size() : 1));
    if (!rows.empty()) BBFMM_CUDA_OK(cudaMemcpy(*dst, rows.data(), sizeof(int64_t) * rows.size(), cudaMemcpyHostToDevice));
    return BBFMM_OK;
  };
  for (int l = m2l_first; l <= maxlev; ++l) {
    TRY(upload(src_runs, l, &src_list[l], &n_src[l]));
    TRY(upload(tgt_runs, l, &tgt_list[l], &n_tgt[l]));
  }
  return BBFMM_OK;
}

// Active blocks of parent cells of every level above the region level, the tiles of the M2L
// kernels under a target region: a block is active when one of its cells descends from an
// active region cell. The FP64 / FP32 kernels take 2 x 2 x 2 blocks, 8 per tile. The
// tensor-core kernel takes 2 x 2 x 2 blocks (32 per tile) or 4 x 4 x 2 blocks (8 per tile),
// whichever costs less by a model of its tiles: a tile's tensor-core mainloop against the TMA
// requests of its box loads (two per block and stage), of which about 22 fit in the mainloop's
// time (measured: 32 blocks of 2 x 2 x 2 per tile run 3x slower than one 8 x 8 x 4 box).
// Morton order of the blocks within each set.
template <typename T>
int Solver<T>::build_region_tiles() {
  auto blocks = [&](int l, int lx, int ly, int lz, std::vector<int4> &bl) {
    const int lp = l - 1, sh = lp - region_level;
    const int nx = (1 << lp) >> lx, ny = (1 << lp) >> ly, nz = (1 << lp) >> lz;
    for (int set = 0; set < nsets; ++set) {
      const unsigned char *mask = region_host.data() + (size_t)set * pow8i(region_level);
      // blocks in Morton order of their corner cell
      std::vector<std::pair<int64_t, int4>> v;
      for (int bz = 0; bz < nz; ++bz)
        for (int by = 0; by < ny; ++by)
          for (int bx = 0; bx < nx; ++bx) {
            bool act = false;
            for (int z = bz << lz; z < (bz + 1) << lz && !act; ++z)
              for (int y = by << ly; y < (by + 1) << ly && !act; ++y)
                for (int x = bx << lx; x < (bx + 1) << lx && !act; ++x)
                  act = mask[(size_t)grid_to_morton(x >> sh, y >> sh, z >> sh, region_level)] != 0;
            if (act) v.push_back({grid_to_morton(bx << lx, by << ly, bz << lz, lp), make_int4(set, bx << lx, by << ly, bz << lz)});
          }
      std::sort(v.begin(), v.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
      for (const auto &e : v) bl.push_back(e.second);
    }
  };
  auto upload = [&](const std::vector<int4> &bl, int4 **dst, int *count) -> int {
    *count = (int)bl.size();
    TRY(dalloc(dst, bl.size() > 0 ? bl.size() : 1));
    if (!bl.empty()) BBFMM_CUDA_OK(cudaMemcpy(*dst, bl.data(), sizeof(int4) * bl.size(), cudaMemcpyHostToDevice));
    return BBFMM_OK;
  };
  for (int l = region_level + 1; l <= maxlev; ++l) {
    std::vector<int4> b2, b4;
    blocks(l, 1, 1, 1, b2);
    TRY(upload(b2, &region_boxes[l], &region_nboxes[l]));
    int geom = 0x111;
    const std::vector<int4> *tc = &b2;
    if ((1 << (l - 1)) >= 4) {  // 4 x 4 x 2 blocks need a class grid of 4 per axis
      blocks(l, 2, 2, 1, b4);
      auto cost = [](size_t nb, int per) {
        const double tiles = (double)((nb + per - 1) / per);
        return tiles * std::max(1.0, (2.0 * per + 2.0) / 22.0);
      };
      if (cost(b4.size(), 8) < cost(b2.size(), 32)) {
        geom = 0x122;
        tc = &b4;
      }
    }
    region_tcgeom[l] = geom;
    TRY(upload(*tc, &region_tcboxes[l], &region_ntcboxes[l]));
  }
  return BBFMM_OK;
}

// The near-field work list of the current tree for tune.p2p_threads threads per CTA (one
// synchronisation: the item count sizes the launch).
template <typename T>
int Solver<T>::build_near_work() {
  if (!near_work) TRY(dalloc((unsigned char **)&near_work, near_work_bytes(N, maxlev, nsets)));
  int flag = 0;
  TRY(near_work_build(N, leaf_start, maxlev, nsets, tune.p2p_threads, near_work, stream, &near_items, &flag,
                      region_mask, region_level));
  if (flag) return bbfmm_set_error(BBFMM_ERR_ARG, "leaf offsets must rise from 0 to N without decreasing");
  near_threads = tune.p2p_threads;
  return BBFMM_OK;
}

// pot[i] = sum_j q_j / r_ij and fld[i] = grad pot at x_i (FMM), caller's order, no target
// factor: the quantities a backward pass needs.
template <typename T>
int Solver<T>::solve_fields(const void *q_dev, void *pot_dev, void *fld_dev) {
  if (!pos4) return bbfmm_set_error(BBFMM_ERR_STATE, "particles not set");
  if (homogen != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "fields are computed for the 1/r kernel");
  if (!Ert) return bbfmm_set_error(BBFMM_ERR_STATE, "operators not set");
  if (!flds) TRY(dalloc(&flds, 3 * (size_t)(N > 0 ? N : 1)));
  kernel_launches = 0;
  if (timing) {  // stage times of this call alone, as solve keeps them
    for (int i = 0; i < ST_COUNT; ++i) stage_ms[i] = 0.f;
    if (!ev[ST_COUNT]) cudaEventCreate(&ev[ST_COUNT]);
    mark(-1, 0);
  }
  TRY(upward(q_dev, sizeof(T) == 8));
  TRY(interaction(m2l_first, maxlev));
  const Tables tb = tables();
  TRY(leaf_down(true));
  TRY(near(phis, flds));
  TRY((launch_scatter_field<T, T>(N, perm, phis, flds, (T *)pot_dev, (T *)fld_dev, stream)));
  mark(ST_SCATTER);
  return BBFMM_OK;
}

// Both far fields one after the other (each through the passes of solve_fields) and one
// near-field pass with both charge vectors: each pair's separation, distance and powers are
// computed once for both (the backward of a recomputing gradient needs pot and field for the
// charges q and g o q). The near-field pass needs only the sorted positions and charges, so it
// runs on a second stream while the second far field runs (in its own output buffers, added
// afterwards; with stage timing on, after it on the solver's stream). Results equal those of
// two solve_fields calls.
template <typename T>
int Solver<T>::solve_fields2(const void *q1_dev, const void *q2_dev, void *pot1_dev, void *fld1_dev, void *pot2_dev,
                             void *fld2_dev) {
  if (!pos4) return bbfmm_set_error(BBFMM_ERR_STATE, "particles not set");
  if (homogen != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "fields are computed for the 1/r kernel");
  if (!Ert) return bbfmm_set_error(BBFMM_ERR_STATE, "operators not set");
  const size_t n1 = N > 0 ? N : 1;
  for (auto pr : {std::make_pair(&flds, 3 * n1), std::make_pair(&phis2, n1), std::make_pair(&flds2, 3 * n1),
                  std::make_pair(&qs2, n1), std::make_pair(&phisn, n1), std::make_pair(&fldsn, 3 * n1)})
    if (!*pr.first) TRY(dalloc(pr.first, pr.second));
  if (!side) BBFMM_CUDA_OK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  for (cudaEvent_t &e : side_ev)
    if (!e) BBFMM_CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  kernel_launches = 0;
  if (timing) {
    for (int i = 0; i < ST_COUNT; ++i) stage_ms[i] = 0.f;
    if (!ev[ST_COUNT]) cudaEventCreate(&ev[ST_COUNT]);
    mark(-1, 0);
  }
  // far field of q1 into (phis2, flds2), and q1 in sorted order kept for the near field
  std::swap(phis, phis2);
  std::swap(flds, flds2);
  int rc = upward(q1_dev, sizeof(T) == 8);
  if (rc == BBFMM_OK) rc = interaction(m2l_first, maxlev);
  if (rc == BBFMM_OK) rc = leaf_down(true);
  std::swap(phis, phis2);
  std::swap(flds, flds2);
  TRY(rc);
  TRY(launch_charges_of<T>(N, pos4, qs2, stream));
  // q2 into pos4, then the near field (pos4's charges q2 into (phisn, fldsn), q1 added to the
  // far field in (phis2, flds2)) beside the far field of q2 into (phis, flds)
  if (sizeof(T) == 8) TRY((launch_gather<T, double>(N, perm, nullptr, (const double *)q2_dev, pos4, stream)));
  else TRY((launch_gather<T, float>(N, perm, nullptr, (const float *)q2_dev, pos4, stream)));
  mark(ST_GATHER);
  if (near_threads != tune.p2p_threads) TRY(build_near_work());
  cudaStream_t ns = timing ? stream : side;
  auto near_pass = [&]() -> int {
    BBFMM_CUDA_OK(cudaMemsetAsync(phisn, 0, sizeof(T) * n1, ns));
    BBFMM_CUDA_OK(cudaMemsetAsync(fldsn, 0, sizeof(T) * 3 * n1, ns));
    return launch_near2(mode, N, pos4, leaf_start, maxlev, near_work, nsets, near_items, near_threads, qs2, phisn,
                        fldsn, phis2, flds2, ns, region_mask, region_level);
  };
  if (!timing) {
    BBFMM_CUDA_OK(cudaEventRecord(side_ev[0], stream));
    BBFMM_CUDA_OK(cudaStreamWaitEvent(side, side_ev[0], 0));
    TRY(near_pass());
    BBFMM_CUDA_OK(cudaEventRecord(side_ev[1], side));
  }
  TRY(upward(nullptr, sizeof(T) == 8));  // pos4 already holds q2
  TRY(interaction(m2l_first, maxlev));
  TRY(leaf_down(true));
  if (timing) TRY(near_pass());
  else BBFMM_CUDA_OK(cudaStreamWaitEvent(stream, side_ev[1], 0));
  mark(ST_P2P);
  // the second vector's potential and field: far + near, one addition per value as near() makes it
  TRY(launch_add<T>(N, phisn, phis, stream));
  TRY(launch_add<T>(3 * (int64_t)N, fldsn, flds, stream));
  TRY((launch_scatter_field<T, T>(N, perm, phis2, flds2, (T *)pot1_dev, (T *)fld1_dev, stream)));
  TRY((launch_scatter_field<T, T>(N, perm, phis, flds, (T *)pot2_dev, (T *)fld2_dev, stream)));
  mark(ST_SCATTER);
  return BBFMM_OK;
}

namespace {
std::mutex g_tune_mutex;
std::map<std::string, std::pair<int, int>> g_tune_cache;  // key -> (kind, groups) or (threads, 0)

int bucket(int64_t v) {  // power-of-two bucket
  int b = 0;
  while (v > 1) { v >>= 1; ++b; }
  return b;
}
}  // namespace

template <typename T>
int Solver<T>::autotune(const void *q_dev, int io_double) {
  if (!pos4) return bbfmm_set_error(BBFMM_ERR_STATE, "particles not set");
  struct TimingOff {  // stage timing off while tuning, restored on every return path
    bool &t;
    const bool was;
    explicit TimingOff(bool &x) : t(x), was(x) { t = false; }
    ~TimingOff() { t = was; }
  } timing_off(timing);
  TRY(upward(q_dev, io_double));
  BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
  for (int l = BBFMM_MINLEV; l <= maxlev; ++l) {
    char key[96];
    snprintf(key, sizeof(key), "m2l/%d/%d/%d/%d", mode, n, l, bucket(cells(l)));
    {
      std::lock_guard<std::mutex> g(g_tune_mutex);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        tune.m2l_kind[l] = it->second.first;
        tune.m2l_groups[l] = it->second.second;
        continue;
      }
    }
    // candidates: (kind, offset groups); only the mixed mode has the tensor-core kind
    std::vector<std::pair<int, int>> cand;
    if (tc_default(l)) cand.push_back({0, 0});
    // the DMMA and the SIMT M2L both split their offsets over groups
    for (int g : {1, 3, 7, 21})
      if (dmma_part_elems(l, nsets, g, r) * (int64_t)sizeof(T) <= ((int64_t)1 << 30)) cand.push_back({1, g});
    float best = 3.4e38f;
    std::pair<int, int> pick = cand[0];
    if (cand.size() > 1) {
      for (auto c : cand) {
        tune.m2l_kind[l] = c.first;
        tune.m2l_groups[l] = c.second;
        TRY(alloc_partials());
        float ms[2] = {0.f, 0.f};
        TRY(time_m2l(l, 1, ms));  // warm
        TRY(time_m2l(l, 3, ms));
        if (ms[0] + ms[1] < best) {
          best = ms[0] + ms[1];
          pick = c;
        }
      }
    }
    tune.m2l_kind[l] = pick.first;
    tune.m2l_groups[l] = pick.second;
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tune_cache[key] = pick;
  }
  TRY(alloc_partials());
  // near field: threads per block
  char key[96];
  snprintf(key, sizeof(key), "p2p/%d/%d/%d", mode, bucket(N), bucket(cells(maxlev)));
  bool cached = false;
  {
    std::lock_guard<std::mutex> g(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      tune.p2p_threads = it->second.first;
      cached = true;
    }
  }
  if (!cached && N > 0) {
    cudaEvent_t a, b;
    BBFMM_CUDA_OK(cudaEventCreate(&a));
    BBFMM_CUDA_OK(cudaEventCreate(&b));
    float best = 3.4e38f;
    int pick = 256;
    int rc = BBFMM_OK;
    for (int th : {64, 128, 256}) {
      tune.p2p_threads = th;
      rc = near(phis, nullptr);  // builds the list for th, warm; phis is scratch that the next solve assigns
      if (rc != BBFMM_OK) break;
      cudaEventRecord(a, stream);
      for (int i = 0; i < 3 && rc == BBFMM_OK; ++i) rc = near(phis, nullptr);
      cudaEventRecord(b, stream);
      cudaEventSynchronize(b);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      if (rc == BBFMM_OK && ms < best) {
        best = ms;
        pick = th;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    TRY(rc);
    tune.p2p_threads = pick;
    std::lock_guard<std::mutex> g(g_tune_mutex);
    g_tune_cache[key] = {pick, 0};
  }
  // the list for the choice now, so that no later (possibly captured) solve rebuilds it
  if (near_threads != tune.p2p_threads) TRY(build_near_work());
  BBFMM_CUDA_OK(cudaStreamSynchronize(stream));
  return BBFMM_OK;
}

template <typename T>
int Solver<T>::copy_multipoles_morton(int level, T *host_out) {
  if (level < BBFMM_MINLEV || level > maxlev) return bbfmm_set_error(BBFMM_ERR_ARG, "level out of range");
  if (nsets != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "multipole copies are per single-set solver");
  T *tmp = nullptr;
  TRY(dalloc(&tmp, (size_t)pow8i(level) * r));
  int rc = launch_morton_cpg<T>(level, r, Mall + Moff[level], tmp, 1, stream);
  if (rc == BBFMM_OK) {
    cudaError_t e = cudaMemcpyAsync(host_out, tmp, sizeof(T) * pow8i(level) * r, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    rc = bbfmm_set_cuda_error(e, "copy multipoles", __FILE__, __LINE__);
  }
  cudaFree(tmp);
  return rc;
}

// The M2L output of one level (L = sum E_k M over the interaction lists, before the post-M2L
// projection and its scale), recomputed from the multipoles of the last solve with the launch
// choices of the solve (the mixed mode's tensor-core kernel writing its full FP64 output), r
// values per cell in the reference's Morton order.
template <typename T>
int Solver<T>::copy_m2l_morton(int level, T *host_out) {
  if (level < BBFMM_MINLEV || level > maxlev) return bbfmm_set_error(BBFMM_ERR_ARG, "level out of range");
  if (nsets != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "M2L copies are per single-set solver");
  if (!pos4 || !Lbuf) return bbfmm_set_error(BBFMM_ERR_STATE, "particles not set");
  const T *Ml = Mall + Moff[level];
  const bool split = tc_m2l(level);
  if (split) {
    const bool fused = lead > 0 && tc_fuses_lead(tcops, tc_products, rk());
    if (lead > 0 && !fused) TRY(m2l_fp(Ml, level, 0, lead, lead_rows));
    TRY(launch_m2l_tc(r, Msplit, Mcells(), Moff[level] / r, tcops, (double *)Lbuf, level, offs, stream, nsets,
                      tc_products, rk(), fused ? (const double *)Ml : nullptr, fused ? (const double *)Ert : nullptr));
  } else {
    TRY(m2l_fp(Ml, level, 0, rk(), rk()));
  }
  T *tmp = nullptr;
  TRY(dalloc(&tmp, (size_t)pow8i(level) * r));
  int rc = launch_morton_cpg<T>(level, r, Lbuf, tmp, 1, stream);
  if (rc == BBFMM_OK) {
    cudaError_t e = cudaMemcpyAsync(host_out, tmp, sizeof(T) * pow8i(level) * r, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    rc = bbfmm_set_cuda_error(e, "copy M2L output", __FILE__, __LINE__);
  }
  cudaFree(tmp);
  return rc;
}

template <typename T>
void Solver<T>::release() {
  for (int l = 0; l <= 10; ++l) {
    if (region_boxes[l]) cudaFree(region_boxes[l]);
    if (region_tcboxes[l]) cudaFree(region_tcboxes[l]);
  }
  free_local();
  if (region_mask) cudaFree(region_mask);
  void *ptrs[] = {offs, perm, leaf_start, near_work, pos4, S[0], S[1], F[0], F[1], Mall, Lbuf, Lpart, Msplit,
                  phis, flds, Ssplit, Lsplit, io_q, io_phi, phis2, flds2, qs2, phisn, fldsn};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (own_ops) {
    void *ops[] = {tkz, cw, kw, Ert, Ecol, Bup, Bdn, kwcol, Bup_lead};
    for (void *p : ops)
      if (p) cudaFree(p);
    if (tcops) tc_free_operators(tcops);
    if (tcproj) tc_free_projections(tcproj);
  }
  if (ev[ST_COUNT]) cudaEventDestroy(ev[ST_COUNT]);
  for (cudaEvent_t e : side_ev)
    if (e) cudaEventDestroy(e);
  if (side) cudaStreamDestroy(side);
  if (own_stream && stream) cudaStreamDestroy(stream);
  *this = Solver<T>();
}

template struct Solver<double>;
template struct Solver<float>;

}  // namespace bbfmm

// ============================================================== handle C-ABI
using bbfmm::Solver;

struct bbfmm_b200_solver {
  int mode;
  Solver<double> *d;
  Solver<float> *f;
};

extern "C" {

const char *bbfmm_b200_last_error(void) { return g_last_error.c_str(); }

int bbfmm_b200_version(void) { return BBFMM_B200_VERSION; }

int bbfmm_b200_create(const bbfmm_b200_config *cfg, const void *U, const void *E, int operators_fp32,
                      bbfmm_b200_solver **out) {
  if (!cfg || !U || !E || !out) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  *out = nullptr;
  const int n = cfg->n, n3 = n * n * n, r = n3 / 2;
  bbfmm_b200_solver *h = new bbfmm_b200_solver();
  h->mode = cfg->mode;
  int rc = BBFMM_OK;
  if (cfg->mode == BBFMM_B200_MODE_S) {
    h->f = new Solver<float>();
    rc = h->f->init(n, cfg->maxlev, cfg->L, cfg->mode, cfg->lead, cfg->lead_rows, cfg->device, (cudaStream_t)cfg->stream);
    if (rc == BBFMM_OK) {
      std::vector<float> tkz(n * n), kw(n3), cw(2 * n * n);
      std::vector<int> kt(343);
      rc = bbfmm_weights<float>(n, tkz.data(), kt.data(), kw.data(), cw.data());
      if (rc == BBFMM_OK) rc = h->f->set_tables(tkz.data(), cw.data(), kw.data());
      std::vector<float> Uf((size_t)n3 * r), Ef((size_t)316 * r * r);
      for (size_t i = 0; i < Uf.size(); ++i) Uf[i] = operators_fp32 ? ((const float *)U)[i] : (float)((const double *)U)[i];
      for (size_t i = 0; i < Ef.size(); ++i) Ef[i] = operators_fp32 ? ((const float *)E)[i] : (float)((const double *)E)[i];
      if (rc == BBFMM_OK) rc = h->f->set_operators(Uf.data(), Ef.data());
    }
  } else {
    h->d = new Solver<double>();
    rc = h->d->init(n, cfg->maxlev, cfg->L, cfg->mode, cfg->lead, cfg->lead_rows, cfg->device, (cudaStream_t)cfg->stream);
    if (rc == BBFMM_OK) {
      std::vector<double> tkz(n * n), kw(n3), cw(2 * n * n);
      std::vector<int> kt(343);
      rc = bbfmm_weights<double>(n, tkz.data(), kt.data(), kw.data(), cw.data());
      if (rc == BBFMM_OK) rc = h->d->set_tables(tkz.data(), cw.data(), kw.data());
      std::vector<double> Ud((size_t)n3 * r), Ed((size_t)316 * r * r);
      for (size_t i = 0; i < Ud.size(); ++i) Ud[i] = operators_fp32 ? ((const float *)U)[i] : ((const double *)U)[i];
      for (size_t i = 0; i < Ed.size(); ++i) Ed[i] = operators_fp32 ? ((const float *)E)[i] : ((const double *)E)[i];
      if (rc == BBFMM_OK) rc = h->d->set_operators(Ud.data(), Ed.data());
    }
  }
  if (rc != BBFMM_OK) {
    bbfmm_b200_destroy(h);
    return rc;
  }
  *out = h;
  return BBFMM_OK;
}

int bbfmm_b200_set_particles(bbfmm_b200_solver *h, int N, const void *xyz) {
  if (!h || (N > 0 && !xyz) || N < 0) return bbfmm_set_error(BBFMM_ERR_ARG, "bad particle arguments");
  if (h->f) {
    Solver<float> &s = *h->f;
    std::vector<int> perm(N > 0 ? N : 1), ls(::pow8i(s.maxlev) + 1);
    int rc = bbfmm_sort_particles<float>(N, (const float *)xyz, (float)s.L, s.maxlev, perm.data(), ls.data());
    if (rc != BBFMM_OK) return rc;
    return s.set_particles_sorted(N, perm.data(), ls.data(), (const float *)xyz);
  }
  Solver<double> &s = *h->d;
  std::vector<int> perm(N > 0 ? N : 1), ls(::pow8i(s.maxlev) + 1);
  int rc = bbfmm_sort_particles<double>(N, (const double *)xyz, s.L, s.maxlev, perm.data(), ls.data());
  if (rc != BBFMM_OK) return rc;
  return s.set_particles_sorted(N, perm.data(), ls.data(), (const double *)xyz);
}

int bbfmm_b200_set_particles_device(bbfmm_b200_solver *h, int N, const void *xyz_dev) {
  if (!h || (N > 0 && !xyz_dev) || N < 0) return bbfmm_set_error(BBFMM_ERR_ARG, "bad particle arguments");
  if (h->f) return h->f->set_particles_device(N, (const float *)xyz_dev);
  return h->d->set_particles_device(N, (const double *)xyz_dev);
}

int bbfmm_b200_solve(bbfmm_b200_solver *h, const void *q_dev, void *phi_dev) {
  if (!h || !q_dev || !phi_dev) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  if (h->f) return h->f->solve(q_dev, phi_dev, 0);
  return h->d->solve(q_dev, phi_dev, 1);
}

int bbfmm_b200_solve_fields(bbfmm_b200_solver *h, const void *q_dev, void *pot_dev, void *field_dev) {
  if (!h || !q_dev || (!pot_dev && !field_dev)) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  if (h->f) return h->f->solve_fields(q_dev, pot_dev, field_dev);
  return h->d->solve_fields(q_dev, pot_dev, field_dev);
}

int bbfmm_b200_solve_fields2(bbfmm_b200_solver *h, const void *q1_dev, const void *q2_dev, void *pot1_dev,
                             void *field1_dev, void *pot2_dev, void *field2_dev) {
  if (!h || !q1_dev || !q2_dev || (!pot1_dev && !field1_dev) || (!pot2_dev && !field2_dev))
    return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  if (h->f) return h->f->solve_fields2(q1_dev, q2_dev, pot1_dev, field1_dev, pot2_dev, field2_dev);
  return h->d->solve_fields2(q1_dev, q2_dev, pot1_dev, field1_dev, pot2_dev, field2_dev);
}

int bbfmm_b200_solve_host(bbfmm_b200_solver *h, const void *q_host, void *phi_host) {
  if (!h || !q_host || !phi_host) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const int N = h->f ? h->f->N : h->d->N;
  const size_t es = h->f ? sizeof(float) : sizeof(double);
  cudaStream_t st = h->f ? h->f->stream : h->d->stream;
  if (N == 0) return BBFMM_OK;
  // device staging kept by the solver (freed when the particles change), so repeated calls do
  // not pay cudaMalloc / cudaFree and the device-wide synchronisation of the latter
  void *&qd = h->f ? h->f->io_q : h->d->io_q;
  void *&pd = h->f ? h->f->io_phi : h->d->io_phi;
  if (!qd && cudaMalloc(&qd, es * N) != cudaSuccess) {
    qd = nullptr;
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation for host solve failed");
  }
  if (!pd && cudaMalloc(&pd, es * N) != cudaSuccess) {
    pd = nullptr;
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation for host solve failed");
  }
  int rc = bbfmm_set_cuda_error(cudaMemcpyAsync(qd, q_host, es * N, cudaMemcpyHostToDevice, st), "h2d q", __FILE__,
                                __LINE__);
  if (rc == BBFMM_OK) rc = bbfmm_b200_solve(h, qd, pd);
  if (rc == BBFMM_OK)
    rc = bbfmm_set_cuda_error(cudaMemcpyAsync(phi_host, pd, es * N, cudaMemcpyDeviceToHost, st), "d2h phi",
                              __FILE__, __LINE__);
  if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(cudaStreamSynchronize(st), "sync", __FILE__, __LINE__);
  return rc;
}

int bbfmm_b200_set_timing(bbfmm_b200_solver *h, int on) {
  if (!h) return bbfmm_set_error(BBFMM_ERR_ARG, "null handle");
  if (h->f) h->f->timing = on != 0;
  else h->d->timing = on != 0;
  return BBFMM_OK;
}

int bbfmm_b200_stage_times(const bbfmm_b200_solver *h, float *ms, int count) {
  if (!h || !ms) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const float *src = h->f ? h->f->stage_ms : h->d->stage_ms;
  for (int i = 0; i < count && i < bbfmm::ST_COUNT; ++i) ms[i] = src[i];
  return h->f ? h->f->kernel_launches : h->d->kernel_launches;
}

int bbfmm_b200_copy_multipoles(bbfmm_b200_solver *h, int level, void *host_out) {
  if (!h || !host_out) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  if (h->f) return h->f->copy_multipoles_morton(level, (float *)host_out);
  return h->d->copy_multipoles_morton(level, (double *)host_out);
}

int bbfmm_b200_set_target_region(bbfmm_b200_solver *h, int level, const unsigned char *active) {
  if (!h) return bbfmm_set_error(BBFMM_ERR_ARG, "null handle");
  return h->f ? h->f->set_target_region(level, active) : h->d->set_target_region(level, active);
}

int bbfmm_b200_set_first_m2l_level(bbfmm_b200_solver *h, int level) {
  if (!h) return bbfmm_set_error(BBFMM_ERR_ARG, "null handle");
  const int maxlev = h->f ? h->f->maxlev : h->d->maxlev;
  if (level < BBFMM_MINLEV || level > maxlev) return bbfmm_set_error(BBFMM_ERR_ARG, "first M2L level in [2, maxlev]");
  return h->f ? h->f->set_m2l_first(level) : h->d->set_m2l_first(level);
}

int bbfmm_b200_copy_m2l(bbfmm_b200_solver *h, int level, void *host_out) {
  if (!h || !host_out) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  if (h->f) return h->f->copy_m2l_morton(level, (float *)host_out);
  return h->d->copy_m2l_morton(level, (double *)host_out);
}

int bbfmm_b200_time_m2l(bbfmm_b200_solver *h, int level, int reps, float *ms) {
  if (!h || !ms) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return h->f ? h->f->time_m2l(level, reps, ms) : h->d->time_m2l(level, reps, ms);
}

int bbfmm_b200_device_status(int clear) {
  const int a = bbfmm::tc_status(clear), b = bbfmm::near_status(clear), c = bbfmm::pass_status(clear);
  return a != 0 ? a : (b != 0 ? b : c);
}

int bbfmm_b200_wait_selftest(unsigned limit) {
  if (limit == 0 || limit > (1u << 24)) return -bbfmm_set_error(BBFMM_ERR_ARG, "limit must be in [1, 2^24]");
  return bbfmm::tc_wait_probe(limit, BBFMM_B200_WAIT_SELFTEST_CODE);
}

int bbfmm_b200_direct(int N, const double *xyz_dev, const double *q_dev, int ntarget, const int *targets_dev,
                      double *out_dev, void *stream) {
  if (N < 0 || ntarget < 0 || (ntarget > 0 && (!xyz_dev || !q_dev || !targets_dev || !out_dev)))
    return bbfmm_set_error(BBFMM_ERR_ARG, "bad direct-sum arguments");
  return bbfmm::launch_direct_fp64(N, xyz_dev, q_dev, ntarget, targets_dev, out_dev, (cudaStream_t)stream);
}

int bbfmm_b200_direct_field(int N, const double *xyz_dev, const double *q_dev, int ntarget, const int *targets_dev,
                            double *pot_dev, double *field_dev, void *stream) {
  if (N < 0 || ntarget < 0 ||
      (ntarget > 0 && (!xyz_dev || !q_dev || !targets_dev || (!pot_dev && !field_dev))))
    return bbfmm_set_error(BBFMM_ERR_ARG, "bad direct-sum arguments");
  return bbfmm::launch_direct_field_fp64(N, xyz_dev, q_dev, ntarget, targets_dev, pot_dev, field_dev,
                                         (cudaStream_t)stream);
}

int bbfmm_b200_set_leaf_slab(bbfmm_b200_solver *h, long long cells) {
  if (!h || cells < 0 || (cells > 0 && cells % 64)) return bbfmm_set_error(BBFMM_ERR_ARG, "slab must be a multiple of 64");
  if (h->f) {
    h->f->slab_request = cells;
    return h->f->pos4 ? h->f->alloc_work() : BBFMM_OK;
  }
  h->d->slab_request = cells;
  return h->d->pos4 ? h->d->alloc_work() : BBFMM_OK;
}

int bbfmm_b200_set_kernel(bbfmm_b200_solver *h, int kernel) {
  if (!h) return bbfmm_set_error(BBFMM_ERR_ARG, "null handle");
  const int hg = bbfmm::kernel_homogen(kernel);
  if (!hg) return bbfmm_set_error(BBFMM_ERR_ARG, "unknown kernel");
  if (h->f) h->f->homogen = hg;
  else h->d->homogen = hg;
  return BBFMM_OK;
}

int bbfmm_b200_set_rank(bbfmm_b200_solver *h, int rank) {
  if (!h) return bbfmm_set_error(BBFMM_ERR_ARG, "null handle");
  const int r = h->f ? h->f->r : h->d->r;
  if (rank != 0 && (rank < 32 || rank > r || rank % 32))
    return bbfmm_set_error(BBFMM_ERR_ARG, "rank must be 0 or a multiple of 32 in [32, r]");
  if (h->f) h->f->rank_eff = rank;
  else h->d->rank_eff = rank;
  return BBFMM_OK;
}

int bbfmm_b200_set_tc_products(bbfmm_b200_solver *h, int nprod) {
  if (!h || (nprod != 0 && nprod != 1 && nprod != 3))
    return bbfmm_set_error(BBFMM_ERR_ARG, "products must be 0 (adaptive), 1 or 3");
  if (h->f) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core products apply to the mixed mode");
  h->d->tc_products = nprod;
  return BBFMM_OK;
}

int bbfmm_b200_autotune(bbfmm_b200_solver *h, const void *q_dev) {
  if (!h || !q_dev) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  return h->f ? h->f->autotune(q_dev, 0) : h->d->autotune(q_dev, 1);
}

int bbfmm_b200_set_tuning(bbfmm_b200_solver *h, const int *info) {
  if (!h || !info) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const int th = info[0];
  if (th != 64 && th != 128 && th != 256) return bbfmm_set_error(BBFMM_ERR_ARG, "P2P threads: 64, 128 or 256");
  for (int l = 0; l <= 10; ++l)
    if (info[1 + l] < 0 || info[1 + l] > 2 || info[12 + l] < 0 || info[12 + l] > bbfmm::DMMA_PARTS)
      return bbfmm_set_error(BBFMM_ERR_ARG, "M2L kind must be 0, 1 or 2 and groups in [0, 21]");
  auto apply = [&](auto &sv) -> int {
    sv.tune.p2p_threads = th;
    for (int l = 0; l <= 10; ++l) {
      sv.tune.m2l_kind[l] = info[1 + l];
      sv.tune.m2l_groups[l] = info[12 + l];
    }
    if (!sv.pos4) return BBFMM_OK;
    if (sv.near_threads != th) TRY(sv.build_near_work());
    return sv.alloc_partials();
  };
  return h->f ? apply(*h->f) : apply(*h->d);
}

int bbfmm_b200_tuning(const bbfmm_b200_solver *h, int *info) {
  if (!h || !info) return bbfmm_set_error(BBFMM_ERR_ARG, "null argument");
  const bbfmm::Tuning &t = h->f ? h->f->tune : h->d->tune;
  info[0] = t.p2p_threads;
  for (int l = 0; l <= 10; ++l) {
    info[1 + l] = t.m2l_kind[l];
    info[12 + l] = t.m2l_groups[l];
  }
  return BBFMM_OK;
}

void *bbfmm_b200_stream(bbfmm_b200_solver *h) {
  if (!h) return nullptr;
  return h->f ? (void *)h->f->stream : (void *)h->d->stream;
}

void bbfmm_b200_destroy(bbfmm_b200_solver *h) {
  if (!h) return;
  if (h->f) { h->f->release(); delete h->f; }
  if (h->d) { h->d->release(); delete h->d; }
  delete h;
}

int bbfmm_b200_weights(int n, int fp32, void *Tkz, int *Ktable, void *Kweights, void *Cweights) {
  if (fp32) return bbfmm_weights<float>(n, (float *)Tkz, Ktable, (float *)Kweights, (float *)Cweights);
  return bbfmm_weights<double>(n, (double *)Tkz, Ktable, (double *)Kweights, (double *)Cweights);
}

int bbfmm_b200_sort_particles(int N, int fp32, const void *xyz, double L, int maxlev, int *perm, int *leaf_start) {
  if (fp32) return bbfmm_sort_particles<float>(N, (const float *)xyz, (float)L, maxlev, perm, leaf_start);
  return bbfmm_sort_particles<double>(N, (const double *)xyz, L, maxlev, perm, leaf_start);
}

}  // extern "C"
