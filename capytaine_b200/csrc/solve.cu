// Library-level frequency solves, LU handles and asynchronous requests.
//
// The whole indirect frequency-solve of capytaine for one body — what
// BEMSolver.solve_all does for the problems of one omega (bem/solver.py:177-207
// per problem, grouped by bem/problems_and_results.py:267-275): assemble S and
// K at k = omega^2 / g (green_functions/delhommeau.py:405-520 ->
// matrices.f90:28-325), factor K (bem/engines.py:300-346), solve every
// radiation and diffraction right-hand side (problems_and_results.py:373-381,
// 440-449), potential S sigma, pressure integration (bodies/bodies.py:238-250)
// and the coefficients (problems_and_results.py:583-592, airy_waves.py:98-102)
// — sequenced here on the device behind plain C calls, so that a host that
// does not run Python can use the engine.  This file only orders the library's
// own kernels (assembly, block LU, refinement, post-processing); every buffer
// it allocates belongs to the call, the LU handle or the context that
// allocated it.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "common.cuh"

namespace bem {
namespace {

constexpr uint32_t kCtxMagic = 0x42454d43u;  // "BEMC"
constexpr uint32_t kLuMagic = 0x42454d4cu;   // "BEML"
constexpr uint32_t kReqMagic = 0x42454d52u;  // "BEMR"
constexpr int kChunk = 16;                   // right-hand sides per refinement call
constexpr double kMixedTol = 1e-10;          // relative residual of the refined solves
constexpr double kFp64Tol = 1e-13;           // float64 solves, accepted up to kMixedTol at the float64 floor
constexpr int kMaxIter = 30;

// Makes a device current for the duration of a call and restores the caller's.
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int dev) {
    status = cudaGetDevice(&prev);
    if (status == cudaSuccess && prev != dev) status = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Device buffers of one call, freed together.
struct Buffers {
  std::vector<void*> ptrs;
  ~Buffers() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T>
  int get(T** out, size_t count, bool zero = false) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaMalloc");
    ptrs.push_back(p);
    if (zero) BEM_CUDA_CHECK(cudaMemset(p, 0, bytes));
    *out = static_cast<T*>(p);
    return BEM_OK;
  }
  template <class T>
  int upload(T** out, const T* host, size_t count) {
    int st = get(out, count);
    if (st) return st;
    BEM_CUDA_CHECK(cudaMemcpy(*out, host, count * sizeof(T), cudaMemcpyHostToDevice));
    return BEM_OK;
  }
};

struct StreamGuard {
  cudaStream_t s = nullptr;
  ~StreamGuard() {
    if (s) cudaStreamDestroy(s);
  }
};

}  // namespace
}  // namespace bem

// Opaque handles of the header.
struct bem_context {
  uint32_t magic;
  int device;
  bem_green_function_params params;
  int nr, nz;
  double* r_dev;
  double* z_dev;
  double* table_dev;
};

struct bem_lu {
  uint32_t magic;
  int device;
  int n, npad, precision;
  void* K;       // unfactored K: n x n (mixed, ld n) or npad x npad (float64, ld npad)
  void* LU;      // float64 factors (npad x npad), or NULL
  void* work;    // LU workspace (1024-byte aligned start for the mixed one)
  void* work_raw;
  int* piv;
  int* info;
  int* err;
};

struct bem_request {
  uint32_t magic;
  std::thread worker;
  std::atomic<int> done{0};
  int status = BEM_OK;
  char message[256] = {0};
  bem_solve_stats stats{};
};

namespace bem {
namespace {

int check_params(const bem_green_function_params* p) {
  if (!p) return set_error(BEM_ERR_INVALID_ARGUMENT, "null Green function parameters");
  if (p->tabulation_nr < 0 || p->tabulation_nz < 0 || !(p->tabulation_rmax > 0.0) || !(p->tabulation_zmin < 0.0) ||
      p->tabulation_nb_integration_points < 3 ||
      (p->tabulation_grid_shape != BEM_GRID_LEGACY && p->tabulation_grid_shape != BEM_GRID_SCALED_NEMOH3) ||
      (p->gf_singularities != BEM_GF_HIGH_FREQ && p->gf_singularities != BEM_GF_LOW_FREQ))
    return set_error(BEM_ERR_INVALID_ARGUMENT,
                     "Green function parameters out of range (gf_singularities high_freq or low_freq)");
  return BEM_OK;
}

bem_assembly_args base_args(const bem_context* ctx, int n, const double* centers, const double* normals,
                            int nv, const double* vertices, const int32_t* faces, const double* areas,
                            const double* radii, int variant) {
  bem_assembly_args a;
  std::memset(&a, 0, sizeof(a));
  a.n = n;
  a.points_dev = centers;  // collocation at the one-point quadrature (the face centres)
  a.dot_normals_dev = normals;
  a.nb_faces = n;
  a.nb_vertices = nv;
  a.vertices_dev = vertices;
  a.faces_dev = faces;
  a.centers_dev = centers;
  a.normals_dev = normals;
  a.areas_dev = areas;
  a.radii_dev = radii;
  a.nb_quad_points = 1;
  a.quad_points_dev = centers;
  a.quad_weights_dev = areas;
  a.tabulation_nb_integration_points = ctx->params.tabulation_nb_integration_points;
  a.tabulation_grid_shape = ctx->params.tabulation_grid_shape;
  a.nr = ctx->table_dev ? ctx->nr : 0;
  a.nz = ctx->table_dev ? ctx->nz : 0;
  a.r_range_dev = ctx->r_dev;
  a.z_range_dev = ctx->z_dev;
  a.table_dev = ctx->table_dev;
  a.table32_dev = nullptr;
  a.wavenumber = 1.0;
  a.free_surface = 0.0;
  a.gf_singularities = variant;
  a.adjoint_double_layer = 1;
  a.early_dot_product = 1;
  a.diagonal_term = 1;
  a.precision = BEM_PREC_FP64;
  a.out_dtype = BEM_DTYPE_C128;
  return a;
}

// Factorisation of `batch` matrices K (the mixed engine reads K as is, n x n
// with leading dimension n; the float64 one factors a padded copy LU of K).
int factor(int precision, void* K, void* LU, int n, int npad, int batch, int* piv, int* info, void* work, int* err,
           cudaStream_t s) {
  if (precision == BEM_PREC_MIXED)
    return bem_clu_factor(K, n, (int64_t)n * n, n, npad, batch, piv, info, work, err, s);
  BEM_CUDA_CHECK(cudaMemcpyAsync(LU, K, (size_t)batch * npad * npad * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  int st = bem_zpad_identity(LU, npad, (int64_t)npad * npad, batch, n, npad, s);
  if (st) return st;
  return bem_zlu_factor(LU, npad, npad, (int64_t)npad * npad, batch, piv, info, work, s);
}

// Solve of nc <= 16 columns (B, X, R: npad rows, ldb, strideB) with the
// factors, refined against K; the mixed solve continues with GMRES
// preconditioned by the same factors when the refinement stops contracting.
int refined_solve(int precision, const void* K, const void* LU, int n, int npad, int batch, void* work,
                  const int* piv, const void* B, void* X, void* R, int64_t ldb, int64_t strideB, int nc,
                  void* ts_work, double* norms, int* err, Buffers& bufs, bem_solve_stats* stats, cudaStream_t s) {
  int iters = 0;
  double resid = 0.0;
  int st;
  if (precision == BEM_PREC_MIXED) {
    st = bem_refine_solve(K, n, (int64_t)n * n, n, npad, batch, work, piv, B, X, R, ldb, strideB, nc, kMixedTol,
                          kMaxIter, ts_work, norms, err, &iters, &resid, s);
    if (st == BEM_ERR_NOT_CONVERGED) {
      stats->escalated_to_gmres += 1;
      const int restart = 20;
      const int64_t gbytes = bem_gmres_workspace_bytes(n, npad, nc, batch, restart);
      if (gbytes < 0) return set_error(BEM_ERR_INVALID_ARGUMENT, "GMRES workspace shape");
      unsigned char* gw = nullptr;
      if ((st = bufs.get(&gw, (size_t)gbytes + 256))) return st;
      void* gwa = (void*)(((uintptr_t)gw + 255) & ~(uintptr_t)255);
      st = bem_gmres_solve(K, n, (int64_t)n * n, n, npad, batch, B, X, ldb, strideB, nc, 0.0, kMixedTol, restart, 10,
                           work, gwa, err, &iters, &resid, s);
    }
  } else {
    st = bem_zlu_refine_solve(K, npad, (int64_t)npad * npad, n, LU, npad, npad, (int64_t)npad * npad, batch, piv,
                              work, B, X, R, ldb, strideB, nc, kFp64Tol, kMaxIter, ts_work, norms, err, &iters,
                              &resid, s);
    if (st == BEM_ERR_NOT_CONVERGED && resid <= kMixedTol) st = BEM_OK;
  }
  stats->iterations = std::max(stats->iterations, iters);
  stats->residual = std::max(stats->residual, resid);
  return st;
}

int solve_frequency_impl(const bem_context* ctx, const bem_mesh_desc* mesh, int nomega, const double* omegas,
                         int ndof, const double* dof_normals, int nhead, const double* headings, double rho,
                         double g, int precision, double* added_mass, double* damping, double* excitation,
                         bem_solve_stats* stats_out) {
  if (!ctx || ctx->magic != kCtxMagic) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_frequency: bad context");
  if (!mesh || mesh->nb_faces <= 0 || mesh->nb_vertices <= 0 || !mesh->vertices || !mesh->faces ||
      !mesh->centers || !mesh->normals || !mesh->areas || !mesh->radii)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_frequency: incomplete mesh description");
  if (nomega <= 0 || !omegas || ndof <= 0 || !dof_normals || nhead < 0 || (nhead > 0 && !headings) ||
      ndof + nhead > 64 || !(rho > 0.0) || !(g > 0.0) || !added_mass || !damping ||
      (nhead > 0 && !excitation) || (precision != BEM_PREC_FP64 && precision != BEM_PREC_MIXED))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_frequency: bad arguments (ndof + nhead <= 64)");
  for (int w = 0; w < nomega; ++w)
    if (!(omegas[w] > 0.0) || !std::isfinite(omegas[w]))
      return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_frequency: angular frequencies must be finite and > 0");
  DeviceGuard dg(ctx->device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  StreamGuard sg;
  BEM_CUDA_CHECK(cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking));
  cudaStream_t s = sg.s;
  Buffers bufs;
  int st;
  const int n = mesh->nb_faces, nv = mesh->nb_vertices;
  const int nrhs = ndof + nhead;
  // singularity variant of delhommeau.py:466-490: panels on the free surface force low_freq
  int variant = ctx->params.gf_singularities;
  for (int i = 0; i < n; ++i)
    if (std::fabs(mesh->centers[3 * i + 2]) < 1e-6) variant = BEM_GF_LOW_FREQ;
  // host-side arrays: dof normal components zero on lid faces, pressure weights
  // -(dof . n) area on hull faces (bodies/bodies.py:238-250)
  std::vector<int32_t> hull(n, 1);
  if (mesh->hull_mask)
    for (int i = 0; i < n; ++i) hull[i] = mesh->hull_mask[i] ? 1 : 0;
  std::vector<double> dofn((size_t)ndof * n), wdof((size_t)ndof * n);
  for (int d = 0; d < ndof; ++d)
    for (int i = 0; i < n; ++i) {
      const double v = hull[i] ? dof_normals[(size_t)d * n + i] : 0.0;
      dofn[(size_t)d * n + i] = v;
      wdof[(size_t)d * n + i] = -v * mesh->areas[i];
    }
  double *vert, *cen, *nrm, *area, *rad, *dofn_d, *wdof_d, *head_d = nullptr;
  int32_t *faces_d, *hull_d;
  if ((st = bufs.upload(&vert, mesh->vertices, (size_t)nv * 3))) return st;
  if ((st = bufs.upload(&faces_d, mesh->faces, (size_t)n * 4))) return st;
  if ((st = bufs.upload(&cen, mesh->centers, (size_t)n * 3))) return st;
  if ((st = bufs.upload(&nrm, mesh->normals, (size_t)n * 3))) return st;
  if ((st = bufs.upload(&area, mesh->areas, (size_t)n))) return st;
  if ((st = bufs.upload(&rad, mesh->radii, (size_t)n))) return st;
  if ((st = bufs.upload(&hull_d, hull.data(), (size_t)n))) return st;
  if ((st = bufs.upload(&dofn_d, dofn.data(), dofn.size()))) return st;
  if ((st = bufs.upload(&wdof_d, wdof.data(), wdof.size()))) return st;
  if (nhead > 0 && (st = bufs.upload(&head_d, headings, (size_t)nhead))) return st;

  // batch of frequencies per pass: as many as fit in half the free memory, at most 16
  const int npad = precision == BEM_PREC_MIXED ? (n + 127) / 128 * 128 : (n + 63) / 64 * 64;
  const double per_matrix =
      precision == BEM_PREC_MIXED
          ? 32.0 * n * n + (double)bem_clu_workspace_bytes(npad, 1)
          : 16.0 * n * n + 32.0 * npad * npad + (double)bem_zlu_workspace_bytes(npad, 1);
  size_t free_b = 0, total_b = 0;
  BEM_CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
  const double budget = 0.5 * (double)free_b - 16.0 * n * n;  // the Rankine part
  if (budget < per_matrix) return set_error(BEM_ERR_OUT_OF_MEMORY, "bem_solve_frequency: not enough device memory");
  const int B = std::max(1, std::min({nomega, 16, (int)(budget / per_matrix)}));

  const size_t kn = precision == BEM_PREC_MIXED ? (size_t)n * n : (size_t)npad * npad;
  double2 *S, *K, *LU = nullptr, *rank, *Bv, *Xv, *Rv, *phi, *F, *FK;
  double *om_d, *k_d, *norms;
  int32_t *piv, *info, *flags;
  unsigned char *work_raw, *ts_work;
  if ((st = bufs.get(&S, (size_t)B * n * n))) return st;
  if ((st = bufs.get(&K, (size_t)B * kn))) return st;
  if (precision == BEM_PREC_FP64 && (st = bufs.get(&LU, (size_t)B * npad * npad))) return st;
  if ((st = bufs.get(&rank, (size_t)n * n))) return st;
  const size_t ld = (size_t)npad * nrhs;  // batch stride of B, X, R
  if ((st = bufs.get(&Bv, (size_t)B * ld, true))) return st;
  if ((st = bufs.get(&Xv, (size_t)B * ld, true))) return st;
  if ((st = bufs.get(&Rv, (size_t)B * ld, true))) return st;
  if ((st = bufs.get(&phi, (size_t)B * n * nrhs))) return st;
  if ((st = bufs.get(&F, (size_t)B * nrhs * ndof))) return st;
  if ((st = bufs.get(&FK, (size_t)B * std::max(nhead, 1) * ndof))) return st;
  if ((st = bufs.get(&om_d, (size_t)B))) return st;
  if ((st = bufs.get(&k_d, (size_t)B))) return st;
  if ((st = bufs.get(&norms, (size_t)2 * B * kChunk + 2, true))) return st;
  if ((st = bufs.get(&piv, (size_t)B * npad))) return st;
  if ((st = bufs.get(&info, (size_t)B, true))) return st;
  if ((st = bufs.get(&flags, 2, true))) return st;  // [err, nan]
  const int64_t wbytes =
      precision == BEM_PREC_MIXED ? bem_clu_workspace_bytes(npad, B) + 1024 : bem_zlu_workspace_bytes(npad, B);
  if ((st = bufs.get(&work_raw, (size_t)wbytes))) return st;
  void* work = precision == BEM_PREC_MIXED ? (void*)(((uintptr_t)work_raw + 1023) & ~(uintptr_t)1023) : work_raw;
  if ((st = bufs.get(&ts_work, (size_t)bem_zgemm_ts_workspace_bytes(n, n, std::min(nrhs, kChunk), B)))) return st;

  bem_assembly_args a = base_args(ctx, n, cen, nrm, nv, vert, faces_d, area, rad, variant);
  a.nan_flag_dev = flags + 1;
  a.wavenumber = omegas[0] * omegas[0] / g;
  a.lds = n;
  a.ldk = precision == BEM_PREC_MIXED ? n : npad;
  a.S_dev = S;
  a.K_dev = K;
  // the wavenumber-independent Rankine part, once for the whole sweep
  if ((st = bem_assemble_rankine_part(&a, rank, n, s))) return st;

  bem_solve_stats stats{};
  std::vector<double2> Fh((size_t)B * nrhs * ndof), FKh((size_t)B * std::max(nhead, 1) * ndof);
  std::vector<double> omh(B), kh(B);
  for (int w0 = 0; w0 < nomega; w0 += B) {
    const int nb = std::min(B, nomega - w0);
    for (int i = 0; i < nb; ++i) {
      omh[i] = omegas[w0 + i];
      kh[i] = omh[i] * omh[i] / g;
    }
    BEM_CUDA_CHECK(cudaMemcpyAsync(om_d, omh.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s));
    BEM_CUDA_CHECK(cudaMemcpyAsync(k_d, kh.data(), nb * sizeof(double), cudaMemcpyHostToDevice, s));
    BEM_CUDA_CHECK(cudaMemsetAsync(flags, 0, 2 * sizeof(int), s));
    // S and K of every frequency of the batch: the wave term once per pair of faces
    if ((st = bem_assemble_wave_symmetric_batched(&a, rank, n, kh.data(), nb, (int64_t)n * n, (int64_t)kn, s)))
      return st;
    if ((st = factor(precision, K, LU, n, npad, nb, piv, info, work, flags, s))) return st;
    BEM_CUDA_CHECK(cudaMemsetAsync(Bv, 0, (size_t)nb * ld * sizeof(double2), s));
    if ((st = bem_build_rhs(n, nb, om_d, k_d, g, INFINITY, ndof, dofn_d, nhead, head_d, cen, nrm, hull_d, Bv, npad,
                            (int64_t)ld, s)))
      return st;
    for (int c0 = 0; c0 < nrhs; c0 += kChunk) {
      const int nc = std::min(kChunk, nrhs - c0);
      const size_t off = (size_t)npad * c0;
      if ((st = refined_solve(precision, K, LU, n, npad, nb, work, piv, Bv + off, Xv + off, Rv + off, npad,
                              (int64_t)ld, nc, ts_work, norms, flags, bufs, &stats, s)))
        return st;
      // potential phi = S sigma (bem/solver.py:197-198)
      if ((st = bem_zgemm_ts(n, n, nc, 1.0, 0.0, S, n, (int64_t)n * n, Xv + off, npad, (int64_t)ld, 0.0, 0.0,
                             phi + (size_t)n * c0, n, (int64_t)n * nrhs, nb, ts_work, s)))
        return st;
    }
    if ((st = bem_integrate_pressure(n, nb, nrhs, ndof, phi, n, (int64_t)n * nrhs, om_d, rho, wdof_d, F, s)))
      return st;
    if (nhead > 0 &&
        (st = bem_froude_krylov(n, nb, ndof, nhead, k_d, rho, g, INFINITY, head_d, cen, wdof_d, FK, s)))
      return st;
    int flags_h[2] = {0, 0};
    std::vector<int> info_h(nb);
    BEM_CUDA_CHECK(cudaMemcpyAsync(Fh.data(), F, (size_t)nb * nrhs * ndof * sizeof(double2), cudaMemcpyDeviceToHost,
                                   s));
    if (nhead > 0)
      BEM_CUDA_CHECK(cudaMemcpyAsync(FKh.data(), FK, (size_t)nb * nhead * ndof * sizeof(double2),
                                     cudaMemcpyDeviceToHost, s));
    BEM_CUDA_CHECK(cudaMemcpyAsync(flags_h, flags, sizeof(flags_h), cudaMemcpyDeviceToHost, s));
    BEM_CUDA_CHECK(cudaMemcpyAsync(info_h.data(), info, nb * sizeof(int), cudaMemcpyDeviceToHost, s));
    BEM_CUDA_CHECK(cudaStreamSynchronize(s));
    if (flags_h[1]) return set_error(BEM_ERR_NAN, "Green function returned a NaN in the interaction matrix");
    for (int i = 0; i < nb; ++i)
      if (info_h[i]) return set_error(BEM_ERR_SINGULAR, "zero pivot in the LU factorisation");
    if (flags_h[0]) return set_error(BEM_ERR_TIMEOUT, "a bounded wait of a block substitution timed out");
    // coefficients: added mass Re(F) / omega^2, damping Im(F) / omega, excitation = diffraction + Froude-Krylov
    for (int i = 0; i < nb; ++i) {
      const int w = w0 + i;
      const double om = omh[i];
      for (int r = 0; r < ndof; ++r)
        for (int d = 0; d < ndof; ++d) {
          const double2 f = Fh[((size_t)i * nrhs + r) * ndof + d];
          added_mass[((size_t)w * ndof + r) * ndof + d] = f.x / (om * om);
          damping[((size_t)w * ndof + r) * ndof + d] = f.y / om;
        }
      for (int h = 0; h < nhead; ++h)
        for (int d = 0; d < ndof; ++d) {
          const double2 dif = Fh[((size_t)i * nrhs + ndof + h) * ndof + d];
          const double2 fk = FKh[((size_t)i * nhead + h) * ndof + d];
          double* e = excitation + 2 * (((size_t)w * nhead + h) * ndof + d);
          e[0] = dif.x + fk.x;
          e[1] = dif.y + fk.y;
        }
    }
  }
  if (stats_out) *stats_out = stats;
  return BEM_OK;
}

}  // namespace
}  // namespace bem

using namespace bem;

extern "C" int bem_context_create(int device, const bem_green_function_params* params, bem_context** out) {
  if (!out) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_context_create: null output");
  *out = nullptr;
  int st = check_params(params);
  if (st) return st;
  int count = 0;
  BEM_CUDA_CHECK(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_context_create: no such device");
  DeviceGuard dg(device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  std::unique_ptr<bem_context> ctx(new bem_context());
  ctx->magic = kCtxMagic;
  ctx->device = device;
  ctx->params = *params;
  ctx->nr = params->tabulation_nr;
  ctx->nz = params->tabulation_nz;
  ctx->r_dev = ctx->z_dev = ctx->table_dev = nullptr;
  if (ctx->nr > 1 && ctx->nz > 1) {
    std::vector<double> r(ctx->nr), z(ctx->nz);
    if ((st = bem_default_r_spacing(ctx->nr, params->tabulation_rmax, params->tabulation_grid_shape, r.data())))
      return st;
    if ((st = bem_default_z_spacing(ctx->nz, params->tabulation_zmin, params->tabulation_grid_shape, z.data())))
      return st;
    BEM_CUDA_CHECK(cudaMalloc(&ctx->r_dev, r.size() * sizeof(double)));
    cudaError_t e = cudaMalloc(&ctx->z_dev, z.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->table_dev, (size_t)ctx->nr * ctx->nz * 5 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->r_dev, r.data(), r.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->z_dev, z.data(), z.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(ctx->r_dev);
      cudaFree(ctx->z_dev);
      cudaFree(ctx->table_dev);
      return set_cuda_error(e, "bem_context_create: tabulation buffers");
    }
    st = bem_construct_tabulation(ctx->r_dev, ctx->nr, ctx->z_dev, ctx->nz, params->tabulation_nb_integration_points,
                                  ctx->table_dev, nullptr);
    if (st == BEM_OK) {
      e = cudaDeviceSynchronize();
      if (e != cudaSuccess) st = set_cuda_error(e, "bem_context_create: tabulation");
    }
    if (st) {
      cudaFree(ctx->r_dev);
      cudaFree(ctx->z_dev);
      cudaFree(ctx->table_dev);
      return st;
    }
  }
  *out = ctx.release();
  return BEM_OK;
}

extern "C" int bem_context_tabulation(const bem_context* ctx, double* r_range_host, double* z_range_host,
                                      double* table_host) {
  if (!ctx || ctx->magic != kCtxMagic || !ctx->table_dev)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_context_tabulation: context without a table");
  DeviceGuard dg(ctx->device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  if (r_range_host)
    BEM_CUDA_CHECK(cudaMemcpy(r_range_host, ctx->r_dev, ctx->nr * sizeof(double), cudaMemcpyDeviceToHost));
  if (z_range_host)
    BEM_CUDA_CHECK(cudaMemcpy(z_range_host, ctx->z_dev, ctx->nz * sizeof(double), cudaMemcpyDeviceToHost));
  if (table_host)
    BEM_CUDA_CHECK(cudaMemcpy(table_host, ctx->table_dev, (size_t)ctx->nr * ctx->nz * 5 * sizeof(double),
                              cudaMemcpyDeviceToHost));
  return BEM_OK;
}

extern "C" int bem_context_set_tabulation(bem_context* ctx, const double* table_host) {
  if (!ctx || ctx->magic != kCtxMagic || !ctx->table_dev || !table_host)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_context_set_tabulation: context without a table");
  DeviceGuard dg(ctx->device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  BEM_CUDA_CHECK(cudaMemcpy(ctx->table_dev, table_host, (size_t)ctx->nr * ctx->nz * 5 * sizeof(double),
                            cudaMemcpyHostToDevice));
  return BEM_OK;
}

extern "C" int bem_solve_frequency(const bem_context* ctx, const bem_mesh_desc* mesh, int nomega,
                                   const double* omegas, int ndof, const double* dof_normals, int nhead,
                                   const double* headings, double rho, double g, int precision, double* added_mass,
                                   double* damping, double* excitation, bem_solve_stats* stats) {
  return solve_frequency_impl(ctx, mesh, nomega, omegas, ndof, dof_normals, nhead, headings, rho, g, precision,
                              added_mass, damping, excitation, stats);
}

extern "C" int bem_lu_factor(const bem_context* ctx, const void* K_dev, int64_t ldk, int n, int precision,
                             bem_lu** out) {
  if (!out) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_lu_factor: null output");
  *out = nullptr;
  if (!ctx || ctx->magic != kCtxMagic || !K_dev || n <= 0 || ldk < n ||
      (precision != BEM_PREC_FP64 && precision != BEM_PREC_MIXED))
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_lu_factor: bad arguments");
  DeviceGuard dg(ctx->device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  std::unique_ptr<bem_lu, int (*)(bem_lu*)> lu(new bem_lu(), [](bem_lu* p) {
    cudaFree(p->K);
    cudaFree(p->LU);
    cudaFree(p->work_raw);
    cudaFree(p->piv);
    cudaFree(p->info);
    cudaFree(p->err);
    delete p;
    return 0;
  });
  std::memset(lu.get(), 0, sizeof(bem_lu));
  lu->magic = kLuMagic;
  lu->device = ctx->device;
  lu->n = n;
  lu->precision = precision;
  const bool mixed = precision == BEM_PREC_MIXED;
  lu->npad = mixed ? (n + 127) / 128 * 128 : (n + 63) / 64 * 64;
  const int npad = lu->npad;
  const int64_t ldK = mixed ? n : npad;
  const int64_t wbytes = mixed ? bem_clu_workspace_bytes(npad, 1) + 1024 : bem_zlu_workspace_bytes(npad, 1);
  BEM_CUDA_CHECK(cudaMalloc(&lu->K, (size_t)ldK * (mixed ? n : npad) * sizeof(double2)));
  if (!mixed) BEM_CUDA_CHECK(cudaMalloc(&lu->LU, (size_t)npad * npad * sizeof(double2)));
  BEM_CUDA_CHECK(cudaMalloc(&lu->work_raw, (size_t)wbytes));
  BEM_CUDA_CHECK(cudaMalloc(&lu->piv, (size_t)npad * sizeof(int)));
  BEM_CUDA_CHECK(cudaMalloc(&lu->info, sizeof(int)));
  BEM_CUDA_CHECK(cudaMalloc(&lu->err, sizeof(int)));
  BEM_CUDA_CHECK(cudaMemset(lu->err, 0, sizeof(int)));
  lu->work = mixed ? (void*)(((uintptr_t)lu->work_raw + 1023) & ~(uintptr_t)1023) : lu->work_raw;
  // the unfactored matrix is kept for the residuals of every solve
  BEM_CUDA_CHECK(cudaMemset(lu->K, 0, (size_t)ldK * (mixed ? n : npad) * sizeof(double2)));
  BEM_CUDA_CHECK(cudaMemcpy2D(lu->K, ldK * sizeof(double2), K_dev, ldk * sizeof(double2), n * sizeof(double2), n,
                              cudaMemcpyDeviceToDevice));
  int st = factor(precision, lu->K, lu->LU, n, npad, 1, lu->piv, lu->info, lu->work, lu->err, nullptr);
  if (st) return st;
  int info = 0;
  BEM_CUDA_CHECK(cudaMemcpy(&info, lu->info, sizeof(int), cudaMemcpyDeviceToHost));
  if (info) return set_error(BEM_ERR_SINGULAR, "bem_lu_factor: zero pivot in the LU factorisation");
  *out = lu.release();
  return BEM_OK;
}

extern "C" int bem_lu_solve(bem_lu* lu, const void* B_dev, int64_t ldb, int nrhs, void* X_dev, int64_t ldx,
                            bem_solve_stats* stats_out) {
  if (!lu || lu->magic != kLuMagic || !B_dev || !X_dev || nrhs <= 0 || ldb < lu->n || ldx < lu->n)
    return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_lu_solve: bad arguments");
  DeviceGuard dg(lu->device);
  if (dg.status != cudaSuccess) return set_cuda_error(dg.status, "cudaSetDevice");
  const int n = lu->n, npad = lu->npad;
  Buffers bufs;
  int st;
  double2 *Bp, *Xp, *Rp;
  double* norms;
  unsigned char* ts;
  const int nc_max = std::min(nrhs, kChunk);
  if ((st = bufs.get(&Bp, (size_t)npad * nc_max, true))) return st;
  if ((st = bufs.get(&Xp, (size_t)npad * nc_max, true))) return st;
  if ((st = bufs.get(&Rp, (size_t)npad * nc_max, true))) return st;
  if ((st = bufs.get(&norms, (size_t)2 * nc_max + 2, true))) return st;
  if ((st = bufs.get(&ts, (size_t)bem_zgemm_ts_workspace_bytes(n, n, nc_max, 1)))) return st;
  BEM_CUDA_CHECK(cudaMemset(lu->err, 0, sizeof(int)));
  bem_solve_stats stats{};
  for (int c0 = 0; c0 < nrhs; c0 += kChunk) {
    const int nc = std::min(kChunk, nrhs - c0);
    BEM_CUDA_CHECK(cudaMemset(Bp, 0, (size_t)npad * nc_max * sizeof(double2)));
    BEM_CUDA_CHECK(cudaMemcpy2D(Bp, npad * sizeof(double2), (const double2*)B_dev + (size_t)c0 * ldb,
                                ldb * sizeof(double2), n * sizeof(double2), nc, cudaMemcpyDeviceToDevice));
    st = refined_solve(lu->precision, lu->K, lu->LU, n, npad, 1, lu->work, lu->piv, Bp, Xp, Rp, npad,
                       (int64_t)npad * nc, nc, ts, norms, lu->err, bufs, &stats, nullptr);
    if (st) return st;
    BEM_CUDA_CHECK(cudaMemcpy2D((double2*)X_dev + (size_t)c0 * ldx, ldx * sizeof(double2), Xp,
                                npad * sizeof(double2), n * sizeof(double2), nc, cudaMemcpyDeviceToDevice));
  }
  int err = 0;
  BEM_CUDA_CHECK(cudaMemcpy(&err, lu->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return set_error(BEM_ERR_TIMEOUT, "a bounded wait of a block substitution timed out");
  if (stats_out) *stats_out = stats;
  return BEM_OK;
}

extern "C" int bem_solve_submit(const bem_context* ctx, const bem_mesh_desc* mesh, int nomega, const double* omegas,
                                int ndof, const double* dof_normals, int nhead, const double* headings, double rho,
                                double g, int precision, double* added_mass, double* damping, double* excitation,
                                bem_request** out) {
  if (!out) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_submit: null output");
  *out = nullptr;
  if (!ctx || ctx->magic != kCtxMagic) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_solve_submit: bad context");
  std::unique_ptr<bem_request> req(new bem_request());
  req->magic = kReqMagic;
  bem_request* r = req.get();
  try {
    r->worker = std::thread([=]() {
      r->status = solve_frequency_impl(ctx, mesh, nomega, omegas, ndof, dof_normals, nhead, headings, rho, g,
                                       precision, added_mass, damping, excitation, &r->stats);
      if (r->status) std::snprintf(r->message, sizeof(r->message), "%s", bem_last_error());
      r->done.store(1, std::memory_order_release);
    });
  } catch (...) {
    return set_error(BEM_ERR_OUT_OF_MEMORY, "bem_solve_submit: no thread for the request");
  }
  *out = req.release();
  return BEM_OK;
}

extern "C" int bem_request_poll(bem_request* req, int wait, bem_solve_stats* stats) {
  if (!req || req->magic != kReqMagic) return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_request_poll: bad request");
  if (!wait && !req->done.load(std::memory_order_acquire)) return BEM_PENDING;
  if (req->worker.joinable()) req->worker.join();
  if (stats) *stats = req->stats;
  if (req->status) return set_error(req->status, req->message);
  return BEM_OK;
}

extern "C" int bem_release(void* handle) {
  if (!handle) return BEM_OK;
  const uint32_t magic = *static_cast<uint32_t*>(handle);
  if (magic == kCtxMagic) {
    bem_context* ctx = static_cast<bem_context*>(handle);
    DeviceGuard dg(ctx->device);
    cudaFree(ctx->r_dev);
    cudaFree(ctx->z_dev);
    cudaFree(ctx->table_dev);
    ctx->magic = 0;
    delete ctx;
    return BEM_OK;
  }
  if (magic == kLuMagic) {
    bem_lu* lu = static_cast<bem_lu*>(handle);
    DeviceGuard dg(lu->device);
    cudaFree(lu->K);
    cudaFree(lu->LU);
    cudaFree(lu->work_raw);
    cudaFree(lu->piv);
    cudaFree(lu->info);
    cudaFree(lu->err);
    lu->magic = 0;
    delete lu;
    return BEM_OK;
  }
  if (magic == kReqMagic) {
    bem_request* req = static_cast<bem_request*>(handle);
    if (req->worker.joinable()) req->worker.join();
    req->magic = 0;
    delete req;
    return BEM_OK;
  }
  return set_error(BEM_ERR_INVALID_ARGUMENT, "bem_release: not a handle of this library");
}
