// The reference's own C entry points, implemented on the device solver.
//
// Exported here as bbfmm_b200_ref_<name>_<d|s> (real = double / float); the shim libraries
// built from reference_shim.c give them the reference's exact names and signatures
// (include/bbfmm_b200_reference.h), so the reference's host objects link unchanged:
//
//   m2l_drv                     m2l_drv.cu:14-93
//   m2l_host_{basic,sibling_blocking,cluster_blocking,ij_blocking}
//                               m2l_host_basic.cu:18-19, m2l_host_sibling_blocking.cu:22-23,
//                               m2l_host_cluster_blocking.cu:29-30, m2l_host_ij_blocking.cu:166-167
//   anotherFMMCompute           anotherFMMCompute.cu:48-85 / anotherFMMCompute.c:3-40
//   anotherUpwardPass           anotherUpwardPass.c:20-571
//   anotherFMMInteraction       anotherFMMInteraction.cu:29-126 / anotherFMMInteraction.c:7952-8167
//   anotherDownwardPass         anotherDownwardPass.cu:41-411 / anotherDownwardPass.c:3-29
//   anotherNearField            anotherNearField.c:219-346
//
// All arrays are the caller's host arrays, as in the reference; every call copies its
// inputs to the device, computes there and copies its outputs back before returning.
// Ownership follows the reference: anotherUpwardPass allocates (*atree)->proxysval,
// anotherFMMInteraction allocates (*atree)->fieldval and frees proxysval, and
// anotherDownwardPass frees fieldval (anotherUpwardPass.c:49-52,569;
// anotherFMMInteraction.cu:49,76; anotherDownwardPassX.c:433). sourceval, which the
// reference allocates and frees inside the upward pass, is never allocated here.
// The tree is the reference's full uniform octree with leaves at maxlev; the neighbour and
// interaction lists are implied by it and are not read (as in the reference's ij scheme).
// Only dof = 1 is supported, as in the reference's GPU code.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "solver.cuh"

template <typename T>
int bbfmm_weights(int n, T *Tkz, int *Ktable, T *Kweights, T *Cweights);

namespace bbfmm {
namespace ref {

// Layouts of the reference's real3, cell and anotherTree (vec234.h, cell.h:10-22 without
// PBC, anotherTree.h:7-20).
template <typename T> struct Real3 { T x, y, z; };
template <typename T> struct Cell {
  int *neighbors, *interaction;
  Real3<T> *center;
  int *fieldsta, *fieldend, *sourcesta, *sourceend;
  int *ineigh, *iinter;
  int pitch_neighbors, pitch_interaction;
};
template <typename T> struct Tree {
  int ncell, minlev, maxlev;
  int *levsta, *levend;
  T *celeng;
  Cell<T> *c;
  T *fieldval, *sourceval, *proxysval;
  int ncell0;
  int Nf, Ns, *fieldlist, *sourcelist;
};

#define TRY(x)                         \
  do {                                 \
    int rc__ = (x);                    \
    if (rc__ != BBFMM_OK) return rc__; \
  } while (0)

template <typename T> constexpr int mode_of() { return sizeof(T) == 8 ? MODE_D : MODE_S; }

static int order_of_rank(int r) { return r == 32 ? 4 : (r == 256 ? 8 : 0); }

// Solver with the caller's (or our own) Chebyshev tables.
template <typename T>
int make_solver(Solver<T> &s, int n, int maxlev, double L0, const T *Tkz, const T *Cw, const T *Kw) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  TRY(s.init(n, maxlev, L0, mode_of<T>(), 0, 0, dev, nullptr));
  // the reference's arrays hold whole levels (fieldval, proxysval): no leaf slabs
  s.slab_request = (int64_t)1 << 62;
  // the caller's tables where given (the reference passes ComputeWeights' output), else ours
  std::vector<T> tkz(n * n), kw(n * n * n), cw(2 * n * n);
  std::vector<int> kt(343);
  TRY(bbfmm_weights<T>(n, tkz.data(), kt.data(), kw.data(), cw.data()));
  if (Tkz) memcpy(tkz.data(), Tkz, sizeof(T) * tkz.size());
  if (Cw) memcpy(cw.data(), Cw, sizeof(T) * cw.size());
  if (Kw) memcpy(kw.data(), Kw, sizeof(T) * kw.size());
  return s.set_tables(tkz.data(), cw.data(), kw.data());
}

template <typename T>
int check_tree(Tree<T> *t, int n, int dof) {
  if (!t || !t->c) return bbfmm_set_error(BBFMM_ERR_ARG, "null tree");
  if (dof != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "only dof = 1 is supported");
  if (n != 4 && n != 8) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  if (t->minlev != BBFMM_MINLEV || t->maxlev < BBFMM_MINLEV || t->maxlev > 10)
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tree must have minlev 2 and maxlev <= 10");
  if (t->ncell != (int)((pow8i(t->maxlev + 1) - 1) / 7))
    return bbfmm_set_error(BBFMM_ERR_ARG, "tree is not the full uniform octree of its maxlev");
  return BBFMM_OK;
}

// Particles of the tree, leaf-sorted with the tree's own fieldlist and leaf ranges.
template <typename T>
int load_particles(Solver<T> &s, Tree<T> *t, const Real3<T> *xyz) {
  const int maxlev = t->maxlev, N = t->Nf;
  const int64_t nl = pow8i(maxlev), A0 = levsta(maxlev);
  std::vector<int> ls(nl + 1);
  for (int64_t k = 0; k < nl; ++k) ls[k] = t->c->fieldsta[A0 + k];
  ls[nl] = N;
  if (N < 0 || (N > 0 && (!t->fieldlist || !xyz)) || ls[0] != 0)
    return bbfmm_set_error(BBFMM_ERR_ARG, "tree particle arrays missing or not starting at leaf 0");
  for (int64_t k = 0; k < nl; ++k)
    if (ls[k + 1] < ls[k] || t->c->fieldend[A0 + k] - t->c->fieldsta[A0 + k] + 1 != ls[k + 1] - ls[k])
      return bbfmm_set_error(BBFMM_ERR_ARG, "leaf particle ranges are not contiguous in leaf order");
  // the device gathers positions and charges through fieldlist: every entry must index a particle
  for (int i = 0; i < N; ++i)
    if (t->fieldlist[i] < 0 || t->fieldlist[i] >= N)
      return bbfmm_set_error(BBFMM_ERR_ARG, "fieldlist entry outside [0, Nf)");
  return s.set_particles_sorted(N, t->fieldlist, ls.data(), reinterpret_cast<const T *>(xyz));
}

template <typename T>
int upload_q(Solver<T> &s, const T *q, T **qd) {
  *qd = nullptr;
  if (cudaMalloc((void **)qd, sizeof(T) * (s.N > 0 ? s.N : 1)) != cudaSuccess)
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation of q failed");
  if (s.N > 0) {
    BBFMM_CUDA_OK(cudaMemcpyAsync(*qd, q, sizeof(T) * s.N, cudaMemcpyHostToDevice, s.stream));
    BBFMM_CUDA_OK(cudaStreamSynchronize(s.stream));
  }
  return BBFMM_OK;
}

// proxysval (host, reference cell order) of levels lo..hi -> device cpg multipoles.
template <typename T>
int upload_multipoles(Solver<T> &s, const T *proxysval, int lo, int hi) {
  T *tmp = nullptr;
  if (cudaMalloc((void **)&tmp, sizeof(T) * pow8i(hi) * s.r) != cudaSuccess)
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation failed");
  int rc = BBFMM_OK;
  for (int l = lo; l <= hi && rc == BBFMM_OK; ++l) {
    cudaError_t e = cudaMemcpyAsync(tmp, proxysval + (size_t)s.r * levsta(l), sizeof(T) * pow8i(l) * s.r,
                                    cudaMemcpyHostToDevice, s.stream);
    rc = bbfmm_set_cuda_error(e, "h2d multipoles", __FILE__, __LINE__);
    if (rc == BBFMM_OK) rc = launch_morton_cpg<T>(l, s.r, tmp, s.Mall + s.Moff[l], 0, s.stream);
    if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(cudaStreamSynchronize(s.stream), "sync", __FILE__, __LINE__);
  }
  cudaStreamSynchronize(s.stream);
  cudaFree(tmp);
  return rc;
}

// Device L (cpg, one level) -> host array in reference cell order.
template <typename T>
int download_level(Solver<T> &s, const T *dev_cpg, int l, int width, T *host) {
  T *tmp = nullptr;
  if (cudaMalloc((void **)&tmp, sizeof(T) * pow8i(l) * width) != cudaSuccess)
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation failed");
  int rc = launch_morton_cpg<T>(l, width, dev_cpg, tmp, 1, s.stream);
  if (rc == BBFMM_OK) {
    cudaError_t e = cudaMemcpyAsync(host + (size_t)width * levsta(l), tmp, sizeof(T) * pow8i(l) * width,
                                    cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    rc = bbfmm_set_cuda_error(e, "d2h level", __FILE__, __LINE__);
  }
  cudaFree(tmp);
  return rc;
}

// ------------------------------------------------------------------------- M2L
// L[r A + i] for cells A of levels lo..hi (assign), M in reference order; seconds of M2L
// kernel time in *secs (the reference's kernel_exec_time).
template <typename T>
int m2l_levels(int lo, int hi, int r, T *L, const T *K, const T *M, double *secs) {
  const int n = order_of_rank(r);
  if (!n) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "rank r must be 32 or 256");
  if (lo < BBFMM_MINLEV || hi < lo || hi > 10) return bbfmm_set_error(BBFMM_ERR_ARG, "bad level range");
  if (!L || !K || !M) return bbfmm_set_error(BBFMM_ERR_ARG, "null array");
  Solver<T> s;
  int rc = make_solver(s, n, hi, 1.0, (const T *)nullptr, (const T *)nullptr, (const T *)nullptr);
  if (rc == BBFMM_OK) rc = s.set_operators(nullptr, K);
  if (rc == BBFMM_OK) rc = s.alloc_work();
  if (rc == BBFMM_OK) rc = upload_multipoles(s, M, lo, hi);
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double tot = 0.0;
  for (int l = lo; l <= hi && rc == BBFMM_OK; ++l) {
    cudaEventRecord(a, s.stream);
    rc = s.m2l_fp(s.Mall + s.Moff[l], l, 0, r, r);
    cudaEventRecord(b, s.stream);
    if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(cudaEventSynchronize(b), "m2l", __FILE__, __LINE__);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    tot += ms * 1e-3;
    if (rc == BBFMM_OK) rc = download_level(s, s.Lbuf, l, r, L);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  s.release();
  if (secs) *secs = tot;
  return rc;
}

// --------------------------------------------------------------------- passes
template <typename T>
int upward(Tree<T> **atree, const Real3<T> *source, const T *Cweights, const T *Tkz, const T *q, const T *V,
           const T *Kweights, int cutoff, int n, int dof) {
  Tree<T> *t = atree ? *atree : nullptr;
  TRY(check_tree(t, n, dof));
  if (cutoff != n * n * n / 2) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "cutoff must be n^3/2");
  Solver<T> s;
  T *qd = nullptr;
  int rc = make_solver(s, n, t->maxlev, (double)t->celeng[0], Tkz, Cweights, Kweights);
  if (rc == BBFMM_OK) rc = s.set_operators(V, nullptr);
  if (rc == BBFMM_OK) rc = load_particles(s, t, source);
  if (rc == BBFMM_OK) rc = upload_q(s, q, &qd);
  if (rc == BBFMM_OK) rc = s.upward(qd, sizeof(T) == 8);
  T *P = nullptr;
  if (rc == BBFMM_OK) {
    P = (T *)malloc(sizeof(T) * (size_t)t->ncell * cutoff);
    if (!P) rc = bbfmm_set_error(BBFMM_ERR_NOMEM, "host allocation of proxysval failed");
  }
  for (int l = BBFMM_MINLEV; l <= t->maxlev && rc == BBFMM_OK; ++l)
    rc = s.copy_multipoles_morton(l, P + (size_t)cutoff * levsta(l));
  if (rc == BBFMM_OK) {
    memset(P, 0, sizeof(T) * (size_t)cutoff * levsta(BBFMM_MINLEV));  // levels 0, 1 unused
    t->proxysval = P;
    t->sourceval = nullptr;
  } else {
    free(P);
  }
  if (qd) cudaFree(qd);
  s.release();
  return rc;
}

// The reference's kernels (bbfmm.c:109-144), told apart by the homogen argument it passes:
// 1 (LAPLACIAN, 1/r), 2 (LAPLACIANFORCE, x/r^3) and 4 (ONEOVERR4, 1/r^4); 0 for any other.
template <typename T>
int kernel_homogen(T homogen) {
  return homogen == (T)1 ? 1 : (homogen == (T)2 ? 2 : (homogen == (T)4 ? 4 : 0));
}

template <typename T>
int interaction(Tree<T> **atree, const T *E, const int *Ktable, const T *U, const T *Kweights, int n, int dof,
                int cutoff, T homogen, double *secs) {
  (void)Ktable;
  Tree<T> *t = atree ? *atree : nullptr;
  TRY(check_tree(t, n, dof));
  if (cutoff != n * n * n / 2) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "cutoff must be n^3/2");
  if (!t->proxysval) return bbfmm_set_error(BBFMM_ERR_STATE, "proxysval missing: run the upward pass first");
  if (!kernel_homogen(homogen))
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "kernels with homogen 1 (1/r), 2 (x/r^3) or 4 (1/r^4) only");
  const int n3 = n * n * n;
  Solver<T> s;
  int rc = make_solver(s, n, t->maxlev, (double)t->celeng[0], (const T *)nullptr, (const T *)nullptr, Kweights);
  s.homogen = kernel_homogen(homogen);
  if (rc == BBFMM_OK) rc = s.set_operators(U, E);
  if (rc == BBFMM_OK) rc = s.alloc_work();
  if (rc == BBFMM_OK) rc = upload_multipoles(s, t->proxysval, BBFMM_MINLEV, t->maxlev);
  T *F = nullptr;
  if (rc == BBFMM_OK) {
    F = (T *)calloc((size_t)t->ncell * n3, sizeof(T));
    if (!F) rc = bbfmm_set_error(BBFMM_ERR_NOMEM, "host allocation of fieldval failed");
  }
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double tot = 0.0;
  for (int l = BBFMM_MINLEV; l <= t->maxlev && rc == BBFMM_OK; ++l) {
    cudaEventRecord(a, s.stream);
    rc = s.m2l_post(l);
    cudaEventRecord(b, s.stream);
    if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(cudaEventSynchronize(b), "m2l", __FILE__, __LINE__);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    tot += ms * 1e-3;
    if (rc == BBFMM_OK) {
      cudaError_t e = cudaMemcpyAsync(F + (size_t)n3 * levsta(l), s.F[l & 1], sizeof(T) * pow8i(l) * n3,
                                      cudaMemcpyDeviceToHost, s.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
      rc = bbfmm_set_cuda_error(e, "d2h fieldval", __FILE__, __LINE__);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc == BBFMM_OK) {
    free(t->proxysval);
    t->proxysval = nullptr;
    t->fieldval = F;
  } else {
    free(F);
  }
  s.release();
  if (secs) *secs = tot;
  return rc;
}

// near: add the near field; far: L2L + L2P from fieldval (which is then freed).
template <typename T>
int downward(Tree<T> **atree, const Real3<T> *field, const T *Cweights, const T *Tkz, const T *q, int n, int dof,
             T *phi, bool far, bool near, T homogen) {
  Tree<T> *t = atree ? *atree : nullptr;
  TRY(check_tree(t, n, dof));
  if (near && !kernel_homogen(homogen))
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "kernels with homogen 1 (1/r), 2 (x/r^3) or 4 (1/r^4) only");
  if (far && !t->fieldval) return bbfmm_set_error(BBFMM_ERR_STATE, "fieldval missing: run the interaction first");
  const int n3 = n * n * n, maxlev = t->maxlev;
  Solver<T> s;
  T *qd = nullptr;
  int rc = make_solver(s, n, maxlev, (double)t->celeng[0], Tkz, Cweights, (const T *)nullptr);
  if (rc == BBFMM_OK) rc = load_particles(s, t, field);  // also sizes the work buffers
  if (rc == BBFMM_OK) rc = upload_q(s, q, &qd);
  if (rc == BBFMM_OK) rc = launch_gather<T, T>(s.N, s.perm, nullptr, qd, s.pos4, s.stream);
  const Tables tb = s.tables();
  if (far) {
    for (int l = BBFMM_MINLEV; l <= maxlev && rc == BBFMM_OK; ++l) {
      cudaError_t e = cudaMemcpyAsync(s.F[l & 1], t->fieldval + (size_t)n3 * levsta(l), sizeof(T) * pow8i(l) * n3,
                                      cudaMemcpyHostToDevice, s.stream);
      rc = bbfmm_set_cuda_error(e, "h2d fieldval", __FILE__, __LINE__);
      if (rc == BBFMM_OK && l > BBFMM_MINLEV) rc = launch_l2l<T>(n, s.F[(l - 1) & 1], s.F[l & 1], l - 1, tb, s.stream);
    }
    if (rc == BBFMM_OK)
      rc = launch_l2p<T>(n, s.pos4, s.leaf_start, maxlev, (T)s.L, tb, s.F[maxlev & 1], s.phis, s.stream);
  } else if (rc == BBFMM_OK && s.N > 0) {
    // the near field adds to the caller's phi: start from it in leaf order
    std::vector<T> ps(s.N);
    for (int i = 0; i < s.N; ++i) ps[i] = phi[t->fieldlist[i]];
    cudaError_t e = cudaMemcpyAsync(s.phis, ps.data(), sizeof(T) * s.N, cudaMemcpyHostToDevice, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    rc = bbfmm_set_cuda_error(e, "h2d phi", __FILE__, __LINE__);
  }
  if (near && rc == BBFMM_OK) {
    s.homogen = kernel_homogen(homogen);
    rc = s.near(s.phis, nullptr);
  }
  if (rc == BBFMM_OK && s.N > 0) {
    std::vector<T> ps(s.N);
    cudaError_t e = cudaMemcpyAsync(ps.data(), s.phis, sizeof(T) * s.N, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    rc = bbfmm_set_cuda_error(e, "d2h phi", __FILE__, __LINE__);
    if (rc == BBFMM_OK)
      for (int i = 0; i < s.N; ++i) phi[t->fieldlist[i]] = ps[i];
  }
  if (rc == BBFMM_OK && far) {
    free(t->fieldval);
    t->fieldval = nullptr;
  }
  if (qd) cudaFree(qd);
  s.release();
  return rc;
}

// Whole solve with one device-resident pass chain.
template <typename T>
int compute(Tree<T> **atree, const Real3<T> *field, const Real3<T> *source, const T *q, const T *K, const T *U,
            const T *Tkz, const int *Ktable, const T *Kweights, const T *Cweights, T homogen, int cutoff, int n,
            int dof, T *phi, double *secs) {
  (void)Ktable;
  Tree<T> *t = atree ? *atree : nullptr;
  TRY(check_tree(t, n, dof));
  if (field != source) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "field points must equal the sources");
  if (cutoff != n * n * n / 2) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "cutoff must be n^3/2");
  if (!kernel_homogen(homogen))
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "kernels with homogen 1 (1/r), 2 (x/r^3) or 4 (1/r^4) only");
  Solver<T> s;
  T *qd = nullptr, *pd = nullptr;
  int rc = make_solver(s, n, t->maxlev, (double)t->celeng[0], Tkz, Cweights, Kweights);
  s.homogen = kernel_homogen(homogen);
  if (rc == BBFMM_OK) rc = s.set_operators(U, K);
  if (rc == BBFMM_OK) rc = load_particles(s, t, source);
  if (rc == BBFMM_OK) rc = upload_q(s, q, &qd);
  if (rc == BBFMM_OK && cudaMalloc((void **)&pd, sizeof(T) * (s.N > 0 ? s.N : 1)) != cudaSuccess)
    rc = bbfmm_set_error(BBFMM_ERR_NOMEM, "device allocation of phi failed");
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  if (rc == BBFMM_OK) {
    cudaEventRecord(a, s.stream);
    rc = s.solve(qd, pd, sizeof(T) == 8);
    cudaEventRecord(b, s.stream);
  }
  if (rc == BBFMM_OK && s.N > 0) {
    cudaError_t e = cudaMemcpyAsync(phi, pd, sizeof(T) * s.N, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
    rc = bbfmm_set_cuda_error(e, "d2h phi", __FILE__, __LINE__);
  }
  float ms = 0.f;
  if (rc == BBFMM_OK) cudaEventElapsedTime(&ms, a, b);
  if (secs) *secs = ms * 1e-3;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (qd) cudaFree(qd);
  if (pd) cudaFree(pd);
  s.release();
  return rc;
}

}  // namespace ref
}  // namespace bbfmm

// ============================================================== exported C-ABI
using namespace bbfmm::ref;

#define API extern "C" __attribute__((visibility("default")))

#define DEFINE_PRECISION(SFX, T)                                                                                  \
  API int bbfmm_b200_ref_m2l_levels_##SFX(int lo, int hi, int r, T *L, T *K, T *M, double *secs) {               \
    return m2l_levels<T>(lo, hi, r, L, K, M, secs);                                                                \
  }                                                                                                               \
  API int bbfmm_b200_ref_upward_##SFX(void *atree, void *source, T *Cweights, T *Tkz, T *q, T *V, T *Kweights,   \
                                      int cutoff, int n, int dof) {                                               \
    return upward<T>((Tree<T> **)atree, (const Real3<T> *)source, Cweights, Tkz, q, V, Kweights, cutoff, n, dof); \
  }                                                                                                               \
  API int bbfmm_b200_ref_interaction_##SFX(void *atree, T *E, int *Ktable, T *U, T *Kweights, int n, int dof,    \
                                           int cutoff, T homogen, double *secs) {                                 \
    return interaction<T>((Tree<T> **)atree, E, Ktable, U, Kweights, n, dof, cutoff, homogen, secs);             \
  }                                                                                                               \
  API int bbfmm_b200_ref_downward_##SFX(void *atree, void *field, void *source, T *Cweights, T *Tkz, T *q, T *U, \
                                        int cutoff, int n, int dof, T homogen, T *phi) {                          \
    (void)source; (void)U; (void)cutoff;                                                                          \
    return downward<T>((Tree<T> **)atree, (const Real3<T> *)field, Cweights, Tkz, q, n, dof, phi, true, true,    \
                       homogen);                                                                                  \
  }                                                                                                               \
  API int bbfmm_b200_ref_downward_far_##SFX(void *atree, void *field, T *Cweights, T *Tkz, T *q, T *U,           \
                                            int cutoff, int n, int dof, T homogen, T *phi) {                      \
    (void)U; (void)cutoff;                                                                                        \
    return downward<T>((Tree<T> **)atree, (const Real3<T> *)field, Cweights, Tkz, q, n, dof, phi, true, false,   \
                       homogen);                                                                                  \
  }                                                                                                               \
  API int bbfmm_b200_ref_near_field_##SFX(void *atree, int dof, T homogen, void *field, void *source, T *phi,    \
                                          T *q) {                                                                 \
    (void)source;                                                                                                 \
    Tree<T> *t = atree ? *(Tree<T> **)atree : nullptr;                                                            \
    if (!t) return bbfmm_set_error(BBFMM_ERR_ARG, "null tree");                                                   \
    const int n = 4; /* the order does not enter the near field */                                                \
    return downward<T>((Tree<T> **)atree, (const Real3<T> *)field, nullptr, nullptr, q, n, dof, phi, false,      \
                       true, homogen);                                                                            \
  }                                                                                                               \
  API int bbfmm_b200_ref_compute_##SFX(void *atree, void *field, void *source, T *q, T *K, T *U, T *Tkz,         \
                                       int *Ktable, T *Kweights, T *Cweights, T homogen, int cutoff, int n,       \
                                       int dof, T *phi, double *secs) {                                           \
    return compute<T>((Tree<T> **)atree, (const Real3<T> *)field, (const Real3<T> *)source, q, K, U, Tkz, Ktable, \
                      Kweights, Cweights, homogen, cutoff, n, dof, phi, secs);                                    \
  }

DEFINE_PRECISION(d, double)
DEFINE_PRECISION(s, float)
