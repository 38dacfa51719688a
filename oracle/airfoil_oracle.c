/*
 * ORACLE -- test infrastructure only.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load this library, and only as the
 * checker; the product (op2-common_b200) never links or calls it.
 *
 * Plain C restatement of the reference's Airfoil hot path:
 *   kernels   apps/c/airfoil/airfoil_plain/dp/save_soln.h:1-4, adt_calc.h:1-27,
 *             res_calc.h:1-33, bres_calc.h:1-35, update.h:1-19
 *   loops     op2/include/op_seq.h: every op_par_loop visits n = 0..size-1 in
 *             order, gathers through map[idx + n*dim] (op_arg_set, :30-51),
 *             and op_arg_idx passes n (:38-43)
 *   driver    apps/c/airfoil/airfoil_plain/dp/airfoil.cpp:221-297: save_soln,
 *             then twice {adt_calc, res_calc, bres_calc, update} with rms,
 *             maxerr, errloc reset before each update; rms of the second
 *             update is finalised as sqrt(rms/ncell)
 *
 * The arithmetic keeps the reference's expression trees and float-literal
 * promotions (1.0f, 0.5f as doubles) so that, compiled with
 * -ffp-contract=off, every value is bit-identical to the reference's own
 * sequential build compiled the same way (pinned in tests/test_oracle.py
 * against oracle/_ref/ref_airfoil_seq_strict and tests/golden/).
 *
 * Constants vector k[8] = {gam, gm1, cfl, eps, qinf[0..3]}.
 *
 * The same kernels are instantiated for float storage (suffix _f32): the
 * mixed-precision form computes fluxes in float and keeps the update, rms and
 * maxerr in double (orc_update_mixed).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>

#define SQRT sqrt
#define SQRT_f32 sqrtf
#define FABS fabs
#define FABS_f32 fabsf

#define ORC_KERNELS(T, S)                                                      \
  static void k_adt_calc##S(const T *x1, const T *x2, const T *x3,             \
                            const T *x4, const T *q, T *adt, const T *k) {     \
    const T gam = k[0], gm1 = k[1], cfl = k[2];                                \
    T dx, dy, ri, u, v, c;                                                     \
    ri = (T)1.0f / q[0];                                                       \
    u = ri * q[1];                                                             \
    v = ri * q[2];                                                             \
    c = SQRT##S(gam * gm1 * (ri * q[3] - (T)0.5f * (u * u + v * v)));             \
    dx = x2[0] - x1[0];                                                        \
    dy = x2[1] - x1[1];                                                        \
    *adt = FABS##S(u * dy - v * dx) + c * SQRT##S(dx * dx + dy * dy);                \
    dx = x3[0] - x2[0];                                                        \
    dy = x3[1] - x2[1];                                                        \
    *adt += FABS##S(u * dy - v * dx) + c * SQRT##S(dx * dx + dy * dy);               \
    dx = x4[0] - x3[0];                                                        \
    dy = x4[1] - x3[1];                                                        \
    *adt += FABS##S(u * dy - v * dx) + c * SQRT##S(dx * dx + dy * dy);               \
    dx = x1[0] - x4[0];                                                        \
    dy = x1[1] - x4[1];                                                        \
    *adt += FABS##S(u * dy - v * dx) + c * SQRT##S(dx * dx + dy * dy);               \
    *adt = (*adt) / cfl;                                                       \
  }                                                                            \
                                                                               \
  static void k_res_calc##S(const T *x1, const T *x2, const T *q1,             \
                            const T *q2, const T *adt1, const T *adt2,         \
                            T *res1, T *res2, const T *k) {                    \
    const T gm1 = k[1], eps = k[3];                                            \
    T dx, dy, mu, ri, p1, vol1, p2, vol2, f;                                   \
    dx = x1[0] - x2[0];                                                        \
    dy = x1[1] - x2[1];                                                        \
    ri = (T)1.0f / q1[0];                                                      \
    p1 = gm1 * (q1[3] - (T)0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));       \
    vol1 = ri * (q1[1] * dy - q1[2] * dx);                                     \
    ri = (T)1.0f / q2[0];                                                      \
    p2 = gm1 * (q2[3] - (T)0.5f * ri * (q2[1] * q2[1] + q2[2] * q2[2]));       \
    vol2 = ri * (q2[1] * dy - q2[2] * dx);                                     \
    mu = (T)0.5f * ((*adt1) + (*adt2)) * eps;                                  \
    f = (T)0.5f * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);        \
    res1[0] += f;                                                              \
    res2[0] -= f;                                                              \
    f = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) +          \
        mu * (q1[1] - q2[1]);                                                  \
    res1[1] += f;                                                              \
    res2[1] -= f;                                                              \
    f = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) +          \
        mu * (q1[2] - q2[2]);                                                  \
    res1[2] += f;                                                              \
    res2[2] -= f;                                                              \
    f = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) +                \
        mu * (q1[3] - q2[3]);                                                  \
    res1[3] += f;                                                              \
    res2[3] -= f;                                                              \
  }                                                                            \
                                                                               \
  static void k_bres_calc##S(const T *x1, const T *x2, const T *q1,            \
                             const T *adt1, T *res1, const int *bound,         \
                             const T *k) {                                     \
    const T gm1 = k[1], eps = k[3];                                            \
    const T *qinf = k + 4;                                                     \
    T dx, dy, mu, ri, p1, vol1, p2, vol2, f;                                   \
    dx = x1[0] - x2[0];                                                        \
    dy = x1[1] - x2[1];                                                        \
    ri = (T)1.0f / q1[0];                                                      \
    p1 = gm1 * (q1[3] - (T)0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));       \
    if (*bound == 1) {                                                         \
      res1[1] += +p1 * dy;                                                     \
      res1[2] += -p1 * dx;                                                     \
    } else {                                                                   \
      vol1 = ri * (q1[1] * dy - q1[2] * dx);                                   \
      ri = (T)1.0f / qinf[0];                                                  \
      p2 = gm1 *                                                               \
           (qinf[3] - (T)0.5f * ri * (qinf[1] * qinf[1] + qinf[2] * qinf[2])); \
      vol2 = ri * (qinf[1] * dy - qinf[2] * dx);                               \
      mu = (*adt1) * eps;                                                      \
      f = (T)0.5f * (vol1 * q1[0] + vol2 * qinf[0]) + mu * (q1[0] - qinf[0]);  \
      res1[0] += f;                                                            \
      f = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * qinf[1] + p2 * dy) +      \
          mu * (q1[1] - qinf[1]);                                              \
      res1[1] += f;                                                            \
      f = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * qinf[2] - p2 * dx) +      \
          mu * (q1[2] - qinf[2]);                                              \
      res1[2] += f;                                                            \
      f = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (qinf[3] + p2)) +            \
          mu * (q1[3] - qinf[3]);                                              \
      res1[3] += f;                                                            \
    }                                                                          \
  }                                                                            \
                                                                               \
  void orc_save_soln##S(int ncell, const T *q, T *qold) {                      \
    for (int n = 0; n < ncell; n++)                                            \
      for (int m = 0; m < 4; m++)                                              \
        qold[4 * (size_t)n + m] = q[4 * (size_t)n + m];                        \
  }                                                                            \
                                                                               \
  void orc_adt_calc##S(int ncell, const int *pcell, const T *x, const T *q,    \
                       T *adt, const T *k) {                                   \
    for (int n = 0; n < ncell; n++) {                                          \
      const int *c = pcell + 4 * (size_t)n;                                    \
      k_adt_calc##S(x + 2 * (size_t)c[0], x + 2 * (size_t)c[1],                \
                    x + 2 * (size_t)c[2], x + 2 * (size_t)c[3],                \
                    q + 4 * (size_t)n, adt + n, k);                            \
    }                                                                          \
  }                                                                            \
                                                                               \
  void orc_res_calc##S(int nedge, const int *pedge, const int *pecell,         \
                       const T *x, const T *q, const T *adt, T *res,           \
                       const T *k) {                                           \
    for (int n = 0; n < nedge; n++) {                                          \
      int n1 = pedge[2 * (size_t)n], n2 = pedge[2 * (size_t)n + 1];            \
      int c1 = pecell[2 * (size_t)n], c2 = pecell[2 * (size_t)n + 1];          \
      k_res_calc##S(x + 2 * (size_t)n1, x + 2 * (size_t)n2,                    \
                    q + 4 * (size_t)c1, q + 4 * (size_t)c2, adt + c1,          \
                    adt + c2, res + 4 * (size_t)c1, res + 4 * (size_t)c2, k);  \
    }                                                                          \
  }                                                                            \
                                                                               \
  void orc_bres_calc##S(int nbedge, const int *pbedge, const int *pbecell,     \
                        const int *bound, const T *x, const T *q,              \
                        const T *adt, T *res, const T *k) {                    \
    for (int n = 0; n < nbedge; n++) {                                         \
      int n1 = pbedge[2 * (size_t)n], n2 = pbedge[2 * (size_t)n + 1];          \
      int c1 = pbecell[n];                                                     \
      k_bres_calc##S(x + 2 * (size_t)n1, x + 2 * (size_t)n2,                   \
                     q + 4 * (size_t)c1, adt + c1, res + 4 * (size_t)c1,       \
                     bound + n, k);                                            \
    }                                                                          \
  }

ORC_KERNELS(double, )
ORC_KERNELS(float, _f32)

/* update.h:1-19 through op_seq.h: gbl INC/MAX args point at the caller's
 * variables, op_arg_idx passes n, op_arg_info(&errloc,...,5) is written by the
 * kernel when sqdel beats the running maximum (first index wins ties). */
void orc_update(int ncell, const double *qold, double *q, double *res,
                const double *adt, double *rms, double *maxerr, int *errloc) {
  for (int n = 0; n < ncell; n++) {
    double del, adti;
    adti = 1.0f / adt[n];
    for (int m = 0; m < 4; m++) {
      size_t i = 4 * (size_t)n + m;
      del = adti * res[i];
      q[i] = qold[i] - del;
      res[i] = 0.0f;
      double sqdel = del * del;
      *rms += sqdel;
      if (sqdel > *maxerr) {
        *maxerr = sqdel;
        *errloc = n;
      }
    }
  }
}

/* The mixed-precision update: float storage, the same arithmetic in double. */
void orc_update_mixed(int ncell, const float *qold, float *q, float *res,
                      const float *adt, double *rms, double *maxerr,
                      int *errloc) {
  for (int n = 0; n < ncell; n++) {
    double del, adti;
    adti = 1.0 / (double)adt[n];
    for (int m = 0; m < 4; m++) {
      size_t i = 4 * (size_t)n + m;
      del = adti * (double)res[i];
      q[i] = (float)((double)qold[i] - del);
      res[i] = 0.0f;
      double sqdel = del * del;
      *rms += sqdel;
      if (sqdel > *maxerr) {
        *maxerr = sqdel;
        *errloc = n;
      }
    }
  }
}

/* One Airfoil run of `niter` outer iterations (airfoil.cpp:221-297).
 * q/qold/adt/res are the state (AoS, 4/4/1/4 doubles per cell), updated in
 * place.  Histories (length niter) may be NULL. */
int orc_airfoil_run(int nnode, int ncell, int nedge, int nbedge,
                    const double *x, const int *pcell, const int *pedge,
                    const int *pecell, const int *pbedge, const int *pbecell,
                    const int *bound, double *q, double *qold, double *adt,
                    double *res, const double *k, int niter,
                    double *rms_hist, double *maxerr_hist, int *errloc_hist) {
  (void)nnode;
  for (int iter = 1; iter <= niter; iter++) {
    double rms = 0.0, maxerr = 0.0;
    int errloc = 0;
    orc_save_soln(ncell, q, qold);
    for (int s = 0; s < 2; s++) {
      orc_adt_calc(ncell, pcell, x, q, adt, k);
      orc_res_calc(nedge, pedge, pecell, x, q, adt, res, k);
      orc_bres_calc(nbedge, pbedge, pbecell, bound, x, q, adt, res, k);
      rms = 0.0;
      maxerr = 0.0;
      errloc = 0;
      orc_update(ncell, qold, q, res, adt, &rms, &maxerr, &errloc);
    }
    rms = sqrt(rms / (double)ncell);
    if (rms_hist)
      rms_hist[iter - 1] = rms;
    if (maxerr_hist)
      maxerr_hist[iter - 1] = maxerr;
    if (errloc_hist)
      errloc_hist[iter - 1] = errloc;
  }
  return 0;
}

/* The mixed-precision run: x/q/qold/adt/res in float, k32 the float
 * constants, rms/maxerr in double. */
int orc_airfoil_run_mixed(int ncell, int nedge, int nbedge, const float *x,
                          const int *pcell, const int *pedge,
                          const int *pecell, const int *pbedge,
                          const int *pbecell, const int *bound, float *q,
                          float *qold, float *adt, float *res,
                          const float *k32, int niter, double *rms_hist) {
  for (int iter = 1; iter <= niter; iter++) {
    double rms = 0.0, maxerr = 0.0;
    int errloc = 0;
    orc_save_soln_f32(ncell, q, qold);
    for (int s = 0; s < 2; s++) {
      orc_adt_calc_f32(ncell, pcell, x, q, adt, k32);
      orc_res_calc_f32(nedge, pedge, pecell, x, q, adt, res, k32);
      orc_bres_calc_f32(nbedge, pbedge, pbecell, bound, x, q, adt, res, k32);
      rms = 0.0;
      maxerr = 0.0;
      errloc = 0;
      orc_update_mixed(ncell, qold, q, res, adt, &rms, &maxerr, &errloc);
    }
    if (rms_hist)
      rms_hist[iter - 1] = sqrt(rms / (double)ncell);
  }
  return 0;
}
