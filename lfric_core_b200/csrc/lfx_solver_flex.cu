// Flexible GMRES and GCR (sci_iterative_solver_mod.f90:1055-1237, 1288-1408),
// and the precondition-only, Jacobi and Chebyshev solves (:1664-1694,
// 1745-1815, 1868-1940).
//
// All are written against the abstract-vector operations of the C ABI --
// lfx_vec_{copy,axpy,aypx,scale,set_scalar,dot,norm}, lfx_op_apply and
// lfx_prec_apply -- exactly as the reference writes them against
// abstract_vector_type: every vector operation, apply and preconditioner runs
// on the device, in the same order as the reference, and only the scalars of
// the short recurrences (Hessenberg, Givens, back substitution, GCR
// coefficients) live on the host. Each inner product returns to the host, as
// in the reference. The device operations equal the CPU builtins bit for bit,
// so a solve equals the oracle's or_fgmres / or_gcr bit for bit.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

constexpr double kEps = DBL_EPSILON;  // EPS of constants_mod (epsilon(r_def))

struct Vops {
  int rc = LFX_OK;
  void copy(lfx_vec* d, const lfx_vec* s) {
    if (!rc) rc = lfx_vec_copy(d, s);
  }
  void axpy(lfx_vec* y, double a, const lfx_vec* x) {
    if (!rc) rc = lfx_vec_axpy(y, a, x);
  }
  void aypx(lfx_vec* y, double a, const lfx_vec* x) {
    if (!rc) rc = lfx_vec_aypx(y, a, x);
  }
  void axpby(lfx_vec* z, double a, const lfx_vec* x, double b, const lfx_vec* y) {
    if (!rc) rc = lfx_vec_axpby(z, a, x, b, y);
  }
  void scale(lfx_vec* v, double a) {
    if (!rc) rc = lfx_vec_scale(v, a);
  }
  void set(lfx_vec* v, double c) {
    if (!rc) rc = lfx_vec_set_scalar(v, c);
  }
  double dot(const lfx_vec* a, const lfx_vec* b) {
    double d = 0.0;
    if (!rc) rc = lfx_vec_dot(a, b, &d);
    return d;
  }
  double norm(const lfx_vec* a) {
    double d = 0.0;
    if (!rc) rc = lfx_vec_norm(a, &d);
    return d;
  }
  void A(lfx_op* op, const lfx_vec* x, lfx_vec* y, int32_t* applies) {
    if (!rc) rc = lfx_op_apply(op, x, y);
    ++*applies;
  }
  void P(lfx_prec* p, const lfx_vec* x, lfx_vec* y) {
    if (!rc) rc = lfx_prec_apply(p, x, y);
  }
};

// Givens reduction of the (k+1) x k Hessenberg matrix and back substitution,
// :1153-1182, every a + b*c one fma as in the oracle.
void hessenberg_solve(std::vector<double>& h, std::vector<double>& g, std::vector<double>& u,
                      int k) {
  auto H = [&](int i, int j) -> double& { return h[(i - 1) + (size_t)(k + 1) * (j - 1)]; };
  for (int iv = 1; iv <= k; ++iv) {
    const double nrm = std::sqrt(std::fma(H(iv, iv), H(iv, iv), H(iv + 1, iv) * H(iv + 1, iv)));
    const double si = H(iv + 1, iv) / nrm;
    const double ci = H(iv, iv) / nrm;
    const double p = std::fma(ci, g[iv - 1], si * g[iv]);
    const double q = std::fma(-si, g[iv - 1], ci * g[iv]);
    g[iv - 1] = p;
    g[iv] = q;
    for (int ivj = iv; ivj <= k; ++ivj) {
      const double h1 = std::fma(ci, H(iv, ivj), si * H(iv + 1, ivj));
      const double h2 = std::fma(-si, H(iv, ivj), ci * H(iv + 1, ivj));
      H(iv, ivj) = h1;
      H(iv + 1, ivj) = h2;
    }
  }
  u[k - 1] = g[k - 1] / H(k, k);
  for (int iv = k - 1; iv >= 1; --iv) {
    u[iv - 1] = g[iv - 1];
    for (int ivj = iv + 1; ivj <= k; ++ivj) u[iv - 1] = std::fma(-H(iv, ivj), u[ivj - 1], u[iv - 1]);
    u[iv - 1] = u[iv - 1] / H(iv, iv);
  }
}

}  // namespace

namespace lfx {

// work: s, w, dx, Ax, res, v[gcrk], Pv[gcrk]
int fgmres_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
                const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                lfx_solve_info* info) {
  const int k = cfg.gcrk;
  lfx_vec *s = work[0], *w = work[1], *dx = work[2], *Ax = work[3], *res = work[4];
  const lfx_vec* const* v = work.data() + 5;
  lfx_vec* const* vv = work.data() + 5;
  lfx_vec* const* Pv = work.data() + 5 + k;
  std::vector<double> h((size_t)(k + 1) * k, 0.0), g(k + 1, 0.0), u(k, 0.0);
  auto H = [&](int i, int j) -> double& { return h[(i - 1) + (size_t)(k + 1) * (j - 1)]; };
  Vops o;
  o.set(dx, 0.0);
  o.set(Ax, 0.0);
  o.copy(res, b);  // assumes a zero initial guess (:1087)
  double sc_err = o.norm(res);
  if (o.rc) return o.rc;
  info->initial_norm = sc_err;
  if (sc_err < kEps) {  // :1092-1097, x unchanged
    info->converged = 1;
    info->final_norm = sc_err;
    return LFX_OK;
  }
  if (cfg.monitor_convergence) sc_err = std::fmax(sc_err, cfg.a_tol);
  o.copy(s, res);
  double beta = o.norm(s);
  o.copy(vv[0], s);
  o.scale(vv[0], 1.0 / beta);
  g[0] = beta;
  double err = 0.0;
  int iter;
  for (iter = 1; iter <= cfg.max_iter && !o.rc; ++iter) {
    for (int iv = 1; iv <= k; ++iv) {
      o.P(prec, v[iv - 1], Pv[iv - 1]);
      o.A(op, Pv[iv - 1], s, &info->applies);
      o.copy(w, s);
      for (int ivj = 1; ivj <= iv; ++ivj) {
        H(ivj, iv) = o.dot(v[ivj - 1], w);
        o.axpy(w, -H(ivj, iv), v[ivj - 1]);
      }
      H(iv + 1, iv) = o.norm(w);
      if (iv < k) {
        o.copy(vv[iv], w);
        o.scale(vv[iv], 1.0 / H(iv + 1, iv));
      }
    }
    if (o.rc) break;
    hessenberg_solve(h, g, u, k);
    for (int iv = 1; iv <= k; ++iv) o.axpy(dx, u[iv - 1], Pv[iv - 1]);
    o.A(op, dx, Ax, &info->applies);
    o.copy(res, Ax);
    o.aypx(res, -1.0, b);
    beta = o.norm(res);
    info->iterations = iter;
    info->final_norm = beta;
    if (cfg.monitor_convergence) {
      err = beta / sc_err;
      info->final_rel = err;
      if (err < cfg.r_tol) {
        info->converged = 1;
        break;
      }
    }
    o.copy(s, res);
    o.set(vv[0], 0.0);
    o.axpy(vv[0], 1.0 / beta, s);
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
  }
  if (o.rc) return o.rc;
  if (std::isnan(err) || std::isnan(beta)) info->status = LFX_NAN_DETECTED;
  o.axpy(x, 1.0, dx);  // :1228
  return o.rc;
}

// work: dx, res, Ax, v[gcrk], Pv[gcrk]
int gcr_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
             const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
             lfx_solve_info* info) {
  const int k = cfg.gcrk;
  lfx_vec *dx = work[0], *res = work[1], *Ax = work[2];
  lfx_vec* const* v = work.data() + 3;
  lfx_vec* const* Pv = work.data() + 3 + k;
  Vops o;
  o.set(dx, 0.0);  // :1321-1327
  o.P(prec, b, dx);
  o.A(op, dx, Ax, &info->applies);
  o.copy(res, b);
  o.axpy(res, -1.0, Ax);
  double sc_err = o.norm(b);  // :1330
  if (o.rc) return o.rc;
  info->initial_norm = sc_err;
  if (sc_err < kEps) {
    info->converged = 1;
    info->final_norm = sc_err;
    return LFX_OK;
  }
  if (cfg.monitor_convergence) sc_err = std::fmax(sc_err, cfg.a_tol);
  double err = 0.0, rn = 0.0;
  int iv_final = 0;
  for (int iter = 1; iter <= cfg.max_iter && !o.rc; ++iter) {
    for (int iv = 1; iv <= k; ++iv) {
      o.P(prec, res, Pv[iv - 1]);
      o.A(op, Pv[iv - 1], v[iv - 1], &info->applies);
      for (int ivj = 1; ivj <= iv - 1; ++ivj) {
        const double alpha = o.dot(v[iv - 1], v[ivj - 1]);
        o.axpy(v[iv - 1], -alpha, v[ivj - 1]);
        o.axpy(Pv[iv - 1], -alpha, Pv[ivj - 1]);
      }
      double alpha = o.norm(v[iv - 1]);
      const double beta = 1.0 / alpha;
      o.scale(v[iv - 1], beta);
      o.scale(Pv[iv - 1], beta);
      alpha = o.dot(res, v[iv - 1]);
      o.axpy(dx, alpha, Pv[iv - 1]);
      o.axpy(res, -alpha, v[iv - 1]);
      if (cfg.monitor_convergence) {
        rn = o.norm(res);
        err = rn / sc_err;
        iv_final = iv;
        if (err < cfg.r_tol) break;
      }
    }
    info->iterations = iter;
    info->inner_iterations = iv_final;
    if (cfg.monitor_convergence) {
      info->final_norm = rn;
      info->final_rel = err;
      if (err < cfg.r_tol) {
        info->converged = 1;
        break;
      }
    }
  }
  if (o.rc) return o.rc;
  if (std::isnan(err)) info->status = LFX_NAN_DETECTED;
  o.axpy(x, 1.0, dx);  // :1400
  return o.rc;
}

// work: res, Ax. x = P b; with monitoring, ||b - A x|| against ||b||.
int precondition_only_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
                           const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                           lfx_solve_info* info) {
  lfx_vec *res = work[0], *Ax = work[1];
  Vops o;
  o.P(prec, b, x);
  info->iterations = 1;
  info->converged = 1;
  if (cfg.monitor_convergence) {
    o.copy(res, b);
    const double e0 = o.norm(res);
    o.A(op, x, Ax, &info->applies);
    o.axpy(res, -1.0, Ax);
    const double e = o.norm(res);
    info->initial_norm = e0;
    info->final_norm = e;
    info->final_rel = e / e0;
  }
  return o.rc;
}

// work: r, z. x += -rho P (A x - b), the residual checked before each update.
int jacobi_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg, double rho_relax,
                const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                lfx_solve_info* info) {
  lfx_vec *r = work[0], *z = work[1];
  Vops o;
  o.set(r, 0.0);
  o.set(z, 0.0);
  const double cst = -rho_relax;
  double r_nrm = 0.0, r_nrm_0 = 0.0;
  for (int iter = 1; iter <= cfg.max_iter && !o.rc; ++iter) {
    o.A(op, x, r, &info->applies);
    o.axpy(r, -1.0, b);
    info->iterations = iter;
    if (cfg.monitor_convergence) {
      r_nrm = o.norm(r);
      if (iter == 1) r_nrm_0 = r_nrm;
      info->final_norm = r_nrm;
      info->final_rel = r_nrm / r_nrm_0;
      if (r_nrm / r_nrm_0 <= cfg.r_tol || r_nrm <= cfg.a_tol) {
        info->converged = 1;
        break;
      }
    }
    o.P(prec, r, z);
    o.axpy(x, cst, z);
  }
  info->initial_norm = r_nrm_0;
  if (std::isnan(r_nrm)) info->status = LFX_NAN_DETECTED;
  return o.rc;
}

// work: xp, xo, z, r. max_iter Chebyshev steps from x = 0 for eigenvalue
// bounds [lmin, lmax] of the preconditioned operator.
int chebyshev_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg, double lmin,
                   double lmax, const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                   lfx_solve_info* info) {
  lfx_vec *xp = work[0], *xo = work[1], *z = work[2], *r = work[3];
  Vops o;
  o.set(x, 0.0);
  o.set(xp, 0.0);
  o.set(xo, 0.0);
  double init_norm = 0.0;
  if (cfg.monitor_convergence) init_norm = std::fmax(1.0, o.norm(b));
  const double a1 = 2.0 / (lmax - lmin);
  const double a2 = (lmax + lmin) / (lmax - lmin);
  const double a_over_b = a1 / a2;
  double w = 1.0;
  for (int iter = 1; iter <= cfg.max_iter && !o.rc; ++iter) {
    o.A(op, xo, z, &info->applies);
    o.axpby(r, 1.0, b, -1.0, z);
    o.P(prec, r, z);
    w = 1.0 / (1.0 - w / (4.0 * (a2 * a2)));
    const double wa_over_b = w * a_over_b;
    o.axpby(x, wa_over_b, z, w, xo);
    o.axpy(x, 1.0 - w, xp);
    if (iter < cfg.max_iter) {
      o.copy(xp, xo);
      o.copy(xo, x);
    }
  }
  info->iterations = cfg.max_iter;
  info->converged = 1;
  if (cfg.monitor_convergence) {
    o.A(op, x, z, &info->applies);
    o.axpy(z, -1.0, b);
    const double fn = o.norm(z);
    info->initial_norm = init_norm;
    info->final_norm = fn;
    info->final_rel = fn / init_norm;
    if (std::isnan(fn)) info->status = LFX_NAN_DETECTED;
  }
  return o.rc;
}

}  // namespace lfx
