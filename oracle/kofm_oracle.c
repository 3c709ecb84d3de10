/* kofm_oracle.c - FP64 CPU restatement of the reference's D2Q9 + k-omega
 * time step.  TEST INFRASTRUCTURE (the checker); never linked by the product.
 *
 * Each function names the reference code it restates (paths relative to the
 * reference project).  Arithmetic is FP64 throughout, like the reference
 * (Kernels/Heading.cl:7, FTYPE double).  Deterministic: per-node work is
 * independent, and every reduction sums fixed chunks in a fixed order, so the
 * result does not depend on the OpenMP thread count.
 */
#include "kofm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Direction tables, order C,E,W,N,S,NE,SW,SE,NW (Heading.cl:197-215,
 * clVariablesLB.cpp:953-958). */
static const int CX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
static const int CY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
static const int REV[9] = {0, 2, 1, 4, 3, 6, 5, 8, 7};
static const int BOUND[9] = {0, ORC_E_BOUND, ORC_W_BOUND, ORC_N_BOUND,
                             ORC_S_BOUND, ORC_NE_BOUND, ORC_SW_BOUND,
                             ORC_SE_BOUND, ORC_NW_BOUND};

/* SST constants (Heading.cl:396-410). */
#define KO_BETA_STAR (9. / 100.)
#define KO_SIGMA_K1 0.85
#define KO_SIGMA_K2 1.
#define KO_SIGMA_O1 0.5
#define KO_SIGMA_O2 0.856
#define KO_A1 0.31
#define KO_KAPPA 0.41
#define KO_C_MU_0_25 0.5477225575
#define KO_GAMMA1 (5. / 9.)
#define KO_GAMMA2 0.44

static inline double dmax(double a, double b) { return a < b ? b : a; }
static inline double dmin(double a, double b) { return b < a ? b : a; }

/* ------------------------------------------------------------------------ */
/* Product-form D2Q9 equilibrium (clVariablesLB.cpp:77-117): per axis
 *   phi(0, u) = 2/3 - u^2,   phi(+-1, u) = (1/3 +- u + u^2) / 2,
 * and f_i = rho * phi(cx_i, ux) * phi(cy_i, uy). */
static inline double phi_axis(int c, double u) {
    if (c == 0) return 2. / 3. - u * u;
    return 0.5 * (1. / 3. + (double)c * u + u * u);
}

void orc_feq(double rho, double ux, double uy, double* feq9) {
    for (int q = 0; q < 9; ++q)
        feq9[q] = rho * phi_axis(CX[q], ux) * phi_axis(CY[q], uy);
}

/* ------------------------------------------------------------------------ */
/* One collide + push-stream pass.
 *   komega = 1: LB_collision_SRT_Fluid_w_kOmega (Kernels/lbKernels.cl:345-633)
 *   komega = 0: LB_collision_SRT_Fluid        (Kernels/lbKernels.cl:175-335)
 * Per fluid node (gx < nX):
 *   moments (lbKernels.cl:117-135);
 *   [k-omega] clamp omega<0 -> |omega|, k<0 -> 1e-16 in place (400-410);
 *     F2 and nu_t from the PREVIOUS step's strain rate S (411-420), written
 *     to nut; relaxation rate w = 1/(3(nu_t + nu) + 0.5) (451);
 *   [laminar] w = tau0;
 *   exact-difference forcing with the product-form equilibrium:
 *     f' = f - w (f - feq(rho,u)) - feq(rho,u) + feq(rho, u + (FTERM, 0))
 *     (464-563 / 223-287);
 *   [k-omega] S = -1.5 tau0/rho * sum_i c_i c_i (f_i - feq_i(rho,u)) with the
 *     LAMINAR rate tau0 (581-583);
 *   half-way bounce-back into the node's own reverse slot (166-171) and push
 *   to the neighbours, periodic in x over nX (597-632 / 300-333).
 * The laminar kernel's bound test is "gx > CHANNEL_LENGTH" (lbKernels.cl:189),
 * which also runs padding column nX when nX < XsizeFull; that column and
 * column nX-1 then both push into column 0 (a write race in the reference).
 * The race is not reproducible, so both forms here use gx < nX, which equals
 * the reference whenever nX == XsizeFull (every configuration measured). */
void orc_collide_push(const orc_cfg* c, const double* FA, double* FB,
                      const int16_t* map, double* rho_a, double* ux_a,
                      double* uy_a, double* K, double* O, const double* wallD,
                      double* nut_a, double* Sxy, int options, int komega) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long D = (long)nxf * ny;
#pragma omp parallel for schedule(static)
    for (int gy = 0; gy < ny; ++gy) {
        for (int gx = 0; gx < nx; ++gx) {
            const long gi = gx + (long)nxf * gy;
            const int type = (uint16_t)map[gi];
            if (type & ORC_M_SOLID) continue;
            double f[9];
            for (int q = 0; q < 9; ++q) f[q] = FA[gi + D * q];
            double rho = 0.;
            for (int q = 0; q < 9; ++q) rho += f[q];
            const double inv = 1. / rho;
            const double ux = inv * (f[1] - f[2] + f[5] - f[6] + f[7] - f[8]);
            const double uy = inv * (f[3] - f[4] + f[5] - f[6] - f[7] + f[8]);

            double w = c->tau0;
            if (komega) {
                double om = O[gi], kv = K[gi];
                const double y = wallD[gi];
                if (om < 0.) { om = fabs(om); O[gi] = om; }
                if (kv < 0.) { kv = 1e-16; K[gi] = 1e-16; }
                const double a = 2. * sqrt(kv) / (KO_BETA_STAR * om * y);
                const double b = 500. * c->mu / (y * y * om);
                const double arg = dmax(a, b);
                double F2 = tanh(arg * arg);
                const double sxx = Sxy[gi], sxy = Sxy[gi + D], syy = Sxy[gi + 2 * D];
                F2 *= sqrt(2. * (sxx * sxx + 2. * sxy * sxy + syy * syy));
                const double nut = dmax(
                    dmin(c->max_turb_visc, KO_A1 * kv / dmax(KO_A1 * om, F2)), 1e-16);
                nut_a[gi] = nut;
                w = 1. / (3. * (nut + c->mu) + 0.5);
            }
            if (options & ORC_OPTION_SAVE_MACRO_FIELDS) {
                rho_a[gi] = rho;
                ux_a[gi] = ux + c->fterm / 2.;
                uy_a[gi] = uy;
            }
            double feq[9], feqF[9];
            orc_feq(rho, ux, uy, feq);
            orc_feq(rho, ux + c->fterm, uy, feqF);
            double sxx_n = 0., sxy_n = 0., syy_n = 0.;
            for (int q = 0; q < 9; ++q) {
                const double neq = f[q] - feq[q];
                sxx_n += (double)(CX[q] * CX[q]) * neq;
                sxy_n += (double)(CX[q] * CY[q]) * neq;
                syy_n += (double)(CY[q] * CY[q]) * neq;
                f[q] = f[q] - w * neq - feq[q] + feqF[q];
            }
            if (komega) {
                const double s = -1.5 * c->tau0 / rho;
                Sxy[gi] = s * sxx_n;
                Sxy[gi + D] = s * sxy_n;
                Sxy[gi + 2 * D] = s * syy_n;
            }
            /* push with half-way bounce-back */
            FB[gi] = f[0];
            const int e = (gx < nx - 1) ? 1 : -gx;
            const int wn = (gx > 0) ? -1 : (nx - 1);
            for (int q = 1; q < 9; ++q) {
                if (type & BOUND[q]) {
                    FB[gi + D * REV[q]] = f[q];
                } else {
                    const long dx = CX[q] > 0 ? e : (CX[q] < 0 ? wn : 0);
                    FB[gi + dx + (long)CY[q] * nxf + D * q] = f[q];
                }
            }
        }
    }
}

/* lbIBB (Kernels/lbKernels.cl:640-668): Bouzidi linear interpolated
 * bounce-back on the post-stream buffer, one link per entry of the list
 * (entry = population index of the link direction; q = wall fraction). */
void orc_ibb(const orc_cfg* c, const int32_t* ibb, const double* q, double* FB,
             int n) {
    const long D = (long)c->nxf * c->ny;
    for (int i = 0; i < n; ++i) {
        const long loc = ibb[i];
        const int dir = (int)(loc / D);
        const long node = loc - (long)dir * D;
        const long rev = node + D * REV[dir];
        const double twoQ = 2. * q[i];
        if (twoQ <= 1.0) {
            FB[rev] = twoQ * FB[rev] + (1. - twoQ) * FB[loc];
        } else {
            /* reverse population of the upstream neighbour (Heading.cl:349-356) */
            const long up = node - CX[dir] - (long)CY[dir] * c->nxf;
            const long revNeigh = up + D * REV[dir];
            FB[rev] = 1. / twoQ * (FB[rev] + (twoQ - 1.) * FB[revNeigh]);
        }
    }
}

/* Calc_Ro_J (Kernels/lbKernels.cl:137-164): moments of a population set. */
void orc_macro(const orc_cfg* c, const double* F, const int16_t* map,
               double* rho_a, double* ux_a, double* uy_a) {
    const long D = (long)c->nxf * c->ny;
    for (int gy = 1; gy < c->ny; ++gy)
        for (int gx = 0; gx < c->nxf && gx <= c->nx; ++gx) {
            const long gi = gx + (long)c->nxf * gy;
            if ((uint16_t)map[gi] & ORC_M_SOLID) continue;
            double f[9], rho = 0.;
            for (int q = 0; q < 9; ++q) { f[q] = F[gi + D * q]; rho += f[q]; }
            const double inv = 1. / rho;
            rho_a[gi] = rho;
            ux_a[gi] = inv * (f[1] - f[2] + f[5] - f[6] + f[7] - f[8]);
            uy_a[gi] = inv * (f[3] - f[4] + f[5] - f[6] - f[7] + f[8]);
        }
}

/* ------------------------------------------------------------------------ */
/* Non-uniform 3-point first-derivative weights from link fractions, with the
 * reference's clipping (spacings >= 0.1) and central-difference fallback when
 * |centre weight| > 10 (kOmegaKernels.cl:37-55 and 235-253). */
typedef struct { double e, w, c; } fd3;
static inline void fd_weights(double dpos, double dneg, fd3* d1, fd3* d2) {
    const double a = dmax(dpos, 0.1), b = dmax(dneg, 0.1), s = dmax(a + b, 0.1);
    d1->e = b / (a * s);
    d1->w = -a / (b * s);
    d1->c = (a - b) / (a * b);
    if (fabs(d1->c) > 10.) { d1->e = 1.0 / s; d1->w = -1.0 / s; d1->c = 0.0; }
    if (d2) { d2->e = 2. / (a * s); d2->w = 2. / (b * s); d2->c = -2. / (a * b); }
}

/* Update_kOmega_Diffusivities (Kernels/kOmegaKernels.cl:7-95). */
void orc_komega_diffusivities(const orc_cfg* c, const int16_t* map,
                              const double* K, const double* O,
                              const double* nut, const double* wallD,
                              double* Dk, double* Do, double* F1,
                              double* dkdxy, const double* rho,
                              const double* dX) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long D = (long)nxf * ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const long g = i + (long)nxf * j;
            if ((uint16_t)map[g] & ORC_M_SOLID) continue;
            fd3 X, Y;
            fd_weights(dX[g], dX[g + D], &X, NULL);
            fd_weights(dX[g + 2 * D], dX[g + 3 * D], &Y, NULL);
            const long gw = (i > 0) ? g - 1 : (nx - 1 + (long)j * nxf);
            const long ge = (i < nx - 1) ? g + 1 : ((long)j * nxf);
            const double om = O[g], kv = K[g], y = wallD[g];
            const double dOdx = X.e * O[ge] + X.w * O[gw] + X.c * om;
            const double dKdx = X.e * K[ge] + X.w * K[gw] + X.c * kv;
            const double dOdy = Y.e * O[g + nxf] + Y.w * O[g - nxf] + Y.c * om;
            const double dKdy = Y.e * K[g + nxf] + Y.w * K[g - nxf] + Y.c * kv;
            /* cross-diffusion multipliers 2 sigma_w2 / omega * dk/dx_i */
            const double m = 2. * KO_SIGMA_O2 / om;
            const double mx = m * dKdx, my = m * dKdy;
            dkdxy[g] = mx;
            dkdxy[g + D] = my;
            const double CDkw = dmax(rho[g] * (mx * dOdx + my * dOdy), 1.0e-10);
            double a = dmax(sqrt(kv) / (KO_BETA_STAR * om * y),
                            500. * c->mu / (y * y * om));
            a = dmin(a, 4. * kv * KO_SIGMA_O2 / (CDkw * y * y));
            const double f1 = tanh(pow(a, 4.));
            F1[g] = f1;
            const double nt = nut[g];
            Dk[g] = c->mu + (KO_SIGMA_K1 * f1 + KO_SIGMA_K2 * (1. - f1)) * nt;
            Do[g] = c->mu + (KO_SIGMA_O1 * f1 + KO_SIGMA_O2 * (1. - f1)) * nt;
        }
}

/* Update_kOmega_Coeffs_Implicit (Kernels/kOmegaKernels.cl:187-480):
 * backward-Euler 5-point rows for k and omega with advection velocity
 * J = u - grad(D) (omega adds the cross-diffusion term), production
 * P_k = 2 nu_t S:S - 2/3 k rho tr(S) limited to [0, 10 beta* k omega], each
 * row normalised by its diagonal; fluid nodes next to an E/W/N/S wall get the
 * omega row replaced by omega = min(1000, sqrt(omega_vis^2 + omega_log^2)).
 * Entries are scattered into CSR through the index planes (C,E,W,N,S). */
void orc_komega_coeffs(const orc_cfg* c, const int32_t* ind, const double* K,
                       const double* O, const double* nut, const double* Dk,
                       const double* Do, const double* F1, const double* dkdo,
                       const double* Sxy, const double* rho, const double* ux,
                       const double* uy, double* kA, double* oA, double* kb,
                       double* ob, const double* dX, const double* wallD,
                       const int16_t* map, double dt_in) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long D = (long)nxf * ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const long g = i + (long)nxf * j;
            const int type = (uint16_t)map[g];
            if (type & ORC_M_SOLID) continue;
            double dt = dt_in;
            fd3 X, Y, X2, Y2;
            fd_weights(dX[g], dX[g + D], &X, &X2);
            fd_weights(dX[g + 2 * D], dX[g + 3 * D], &Y, &Y2);
            const long gw = (i > 0) ? g - 1 : (nx - 1 + (long)j * nxf);
            const long ge = (i < nx - 1) ? g + 1 : ((long)j * nxf);
            const double dk = Dk[g], dom = Do[g];
            const double dk_dx = X.e * Dk[ge] + X.w * Dk[gw] + X.c * dk;
            const double do_dx = X.e * Do[ge] + X.w * Do[gw] + X.c * dom;
            const double dk_dy = Y.e * Dk[g + nxf] + Y.w * Dk[g - nxf] + Y.c * dk;
            const double do_dy = Y.e * Do[g + nxf] + Y.w * Do[g - nxf] + Y.c * dom;
            const double Ux = ux[g], Uy = uy[g], Rho = rho[g];
            const double Jxo = Ux - do_dx - dkdo[g];
            const double Jyo = Uy - do_dy - dkdo[g + D];
            const double Jxk = Ux - dk_dx, Jyk = Uy - dk_dy;
            double om = dmax(0.0, O[g]);
            const double kv = dmax(0.0, K[g]);
            const double f1 = F1[g], nt = nut[g];
            const double Sxx = Sxy[g], Sxy_ = Sxy[g + D], Syy = Sxy[g + 2 * D];
            double Pk = 2. * nt * (Sxx * Sxx + Syy * Syy + 2. * Sxy_ * Sxy_) -
                        2. / 3. * kv * Rho * (Sxx + Syy);
            Pk = dmax(dmin(Pk, 10. * KO_BETA_STAR * kv * om), 0.0);
            const double gam = (f1 * KO_GAMMA1 + (1. - f1) * KO_GAMMA2) / nt;
            double Sc = -KO_BETA_STAR * om;

            double Kc = 1. + dt * (Jxk * X.c + Jyk * Y.c - dk * (X2.c + Y2.c)) - Sc;
            double Ke = dt * (Jxk * X.e - dk * X2.e);
            double Kw = dt * (Jxk * X.w - dk * X2.w);
            double Kn = dt * (Jyk * Y.e - dk * Y2.e);
            double Ks = dt * (Jyk * Y.w - dk * Y2.w);
            double Ksrc = kv + dt * Pk;
            const double iKc = 1. / Kc;
            Ke *= iKc; Kw *= iKc; Kn *= iKc; Ks *= iKc; Ksrc *= iKc;

            if (type & ORC_NESW_BOUNDARY) {
                dt = 0.;
                Sc = 0.;
                const double yp = wallD[g];
                const double ovis = (6. * c->mu / 0.075) / (yp * yp);
                const double olog = sqrt(kv) / (KO_C_MU_0_25 * KO_KAPPA * yp);
                om = dmin(1000., sqrt(ovis * ovis + olog * olog));
            }
            double Wc = 1. + dt * (Jxo * X.c + Jyo * Y.c - dom * (X2.c + Y2.c)) - Sc;
            double We = dt * (Jxo * X.e - dom * X2.e);
            double Ww = dt * (Jxo * X.w - dom * X2.w);
            double Wn = dt * (Jyo * Y.e - dom * Y2.e);
            double Ws = dt * (Jyo * Y.w - dom * Y2.w);
            double Wsrc = om + dt * (gam * Pk);
            const double iWc = 1. / Wc;
            We *= iWc; Ww *= iWc; Wn *= iWc; Ws *= iWc; Wsrc *= iWc;

            const long C = ind[g], E = ind[g + D], W = ind[g + 2 * D];
            const long N = ind[g + 3 * D], S = ind[g + 4 * D];
            kA[C] = 1.; oA[C] = 1.;
            kb[g] = Ksrc; ob[g] = Wsrc;
            kA[S] = Ks; kA[W] = Kw; kA[E] = Ke; kA[N] = Kn;
            oA[S] = Ws; oA[W] = Ww; oA[E] = We; oA[N] = Wn;
        }
}

/* ------------------------------------------------------------------------ */
/* CSR pattern of CSR_Inds_Periodic with flags (M_SOLID, M_FLUID,
 * SOLID_BOUNDARY) (SparseMatrix.cpp:57-209 fill_IA/testRow/testNeigh,
 * 369-450 fill_JA; kOmega.h:41).  Rows of solid-boundary nodes hold only the
 * diagonal; other solid rows are empty; fluid rows hold S, then W/C/E in
 * ascending column order under the periodic wrap, then N. */
static int csr_neigh_ok(const orc_cfg* c, const int16_t* map, int i, int j) {
    if (i < 0 || i >= c->nx || j < 0 || j >= c->ny) return 0;
    const int t = (uint16_t)map[i + (long)c->nxf * j];
    return (t & (ORC_SOLID_BOUNDARY | ORC_M_FLUID)) != 0;
}

int orc_csr_build(const orc_cfg* c, const int16_t* map, int32_t* IA,
                  int32_t* JA, int32_t* ind) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long n = (long)nxf * ny;
    enum { iC = 0, iE = 1, iW = 2, iN = 3, iS = 4 };
    int nnz = 0;
    if (IA) IA[0] = 0;
    if (ind) for (long t = 0; t < 5 * n; ++t) ind[t] = -1;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nxf; ++i) {
            const long g = i + (long)nxf * j;
            if (i < nx) {
                const int t = (uint16_t)map[g];
                if (t & ORC_M_SOLID) {
                    if (t & ORC_SOLID_BOUNDARY) {
                        if (JA) JA[nnz] = (int32_t)g;
                        if (ind) ind[g + n * iC] = nnz;
                        ++nnz;
                    }
                } else {
                    const int ie = (i < nx - 1) ? i + 1 : 0;
                    const int iw = (i > 0) ? i - 1 : nx - 1;
                    const int okS = csr_neigh_ok(c, map, i, j - 1);
                    const int okN = csr_neigh_ok(c, map, i, j + 1);
                    const int okE = csr_neigh_ok(c, map, ie, j);
                    const int okW = csr_neigh_ok(c, map, iw, j);
                    int order[3];
                    if (iw < i && i < ie) { order[0] = iW; order[1] = iC; order[2] = iE; }
                    else if (ie < iw && iw < i) { order[0] = iE; order[1] = iW; order[2] = iC; }
                    else { order[0] = iC; order[1] = iE; order[2] = iW; }
                    if (okS) {
                        if (JA) JA[nnz] = (int32_t)(g - nxf);
                        if (ind) ind[g + n * iS] = nnz;
                        ++nnz;
                    }
                    for (int k = 0; k < 3; ++k) {
                        const int d = order[k];
                        if (d == iC) {
                            if (JA) JA[nnz] = (int32_t)g;
                            if (ind) ind[g + n * iC] = nnz;
                            ++nnz;
                        } else if (d == iE && okE) {
                            if (JA) JA[nnz] = (int32_t)(ie + (long)nxf * j);
                            if (ind) ind[g + n * iE] = nnz;
                            ++nnz;
                        } else if (d == iW && okW) {
                            if (JA) JA[nnz] = (int32_t)(iw + (long)nxf * j);
                            if (ind) ind[g + n * iW] = nnz;
                            ++nnz;
                        }
                    }
                    if (okN) {
                        if (JA) JA[nnz] = (int32_t)(g + nxf);
                        if (ind) ind[g + n * iN] = nnz;
                        ++nnz;
                    }
                }
            }
            if (IA) IA[g + 1] = nnz;
        }
    return nnz;
}

void orc_csr_fill_solid_boundary(const orc_cfg* c, const int16_t* map,
                                 const int32_t* ind, double* A) {
    const long n = (long)c->nxf * c->ny;
    for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const long g = i + (long)c->nxf * j;
            if ((uint16_t)map[g] & ORC_SOLID_BOUNDARY) A[ind[g]] = 1.;
        }
    (void)n;
}

/* ------------------------------------------------------------------------ */
/* Deterministic reductions: fixed 128 chunks (the reference's 128 work-groups
 * of normVCL, gmresKernels.cl:5-31), each summed in order, then chunk sums
 * summed in order. */
#define ORC_CHUNKS 128
static double dot_chunked(const double* a, const double* b, long n) {
    double part[ORC_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) {
        const long s = (long)((cidx * (double)n) / ORC_CHUNKS);
        const long e = (long)(((cidx + 1) * (double)n) / ORC_CHUNKS);
        double acc = 0.;
        for (long t = s; t < e; ++t) acc += a[t] * b[t];
        part[cidx] = acc;
    }
    double sum = 0.;
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) sum += part[cidx];
    return sum;
}

static void spmv(int n, const int32_t* IA, const int32_t* JA, const double* A,
                 const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n; ++r) {
        double s = 0.;
        for (int k = IA[r]; k < IA[r + 1]; ++k) s += A[k] * x[JA[k]];
        y[r] = s;
    }
}

/* GMRESSolver::solve (GMRESSolver.cpp:227-355) with the kernels it enqueues
 * (gmresKernels.cl:33-279 prod / Gram-Schmidt / normalise / update,
 * 353-491 updateRHS / updateResidual; GMRESGenerator.cpp:155-200 residual
 * scaling and initial-guess add) and fillArraysWithInitialValues /
 * checkConvergence (GMRESSolver.cpp:1518-1560).  Algorithm: restarted
 * "simpler GMRES" (Walker & Zhou 1994) on the correction system
 * A d = b - A x0 with classical Gram-Schmidt, lazy truncation tests on R and
 * on xi, the rho *= sin(acos(xi/rho)) residual estimator, and x = x0 + d. */
void orc_gmres_solve(int n, const int32_t* IA, const int32_t* JA,
                     const double* A, double* b, double* x, int K,
                     int max_iters, double rel_tol, double abs_tol,
                     orc_gmres_stats* st) {
    double* res = (double*)malloc(sizeof(double) * n);
    double* x0 = (double*)malloc(sizeof(double) * n);
    double* V = (double*)malloc(sizeof(double) * (size_t)n * K);
    double* tmp = (double*)malloc(sizeof(double) * n);
    double R[64 * 64];
    double xi[64], h[64];
    memset(R, 0, sizeof(R));
    memset(xi, 0, sizeof(xi));
    memset(st, 0, sizeof(*st));

    /* updateRHS: b -= A x0 */
    spmv(n, IA, JA, A, x, tmp);
    for (int r = 0; r < n; ++r) b[r] -= tmp[r];
    /* fillArraysWithInitialValues */
    memcpy(res, b, sizeof(double) * n);
    memcpy(x0, x, sizeof(double) * n);
    memset(x, 0, sizeof(double) * n);
    double rho0 = sqrt(dot_chunked(res, res, n));
    const double norm_rhs = rho0;
    st->norm_rhs = norm_rhs;
    double rho = 1.0;
    int iters = 0;
    const int max_restarts = max_iters / K;

    for (int rc = 0; rc < max_restarts; ++rc) {
        if (rc > 0) {
            spmv(n, IA, JA, A, x, tmp);
            for (int r = 0; r < n; ++r) res[r] = b[r] - tmp[r];
            rho0 = sqrt(dot_chunked(res, res, n));
        }
        for (int r = 0; r < n; ++r) res[r] /= rho0;
        rho = 1.0;
        st->restarts = rc + 1;
        /* checkConvergence */
        {
            const double resid = rho0 / norm_rhs;
            if (isnan(resid)) { st->nan = 1; break; }
            if (resid <= rel_tol || rho0 <= abs_tol) break;
        }
        int k;
        for (k = 0; k < K; ++k) {
            double* vk = V + (size_t)k * n;
            const double* src = (k == 0) ? res : V + (size_t)(k - 1) * n;
            spmv(n, IA, JA, A, src, vk);
            if (k > 0) {
                /* classical Gram-Schmidt against v_0..v_{k-1} */
                for (int jv = 0; jv < k; ++jv)
                    h[jv] = dot_chunked(vk, V + (size_t)jv * n, n);
                for (int r = 0; r < n; ++r) {
                    double v = vk[r];
                    for (int jv = 0; jv < k; ++jv) v -= h[jv] * V[(size_t)jv * n + r];
                    vk[r] = v;
                }
                for (int jv = 0; jv < k; ++jv) R[jv + k * K] = h[jv];
            }
            const double nrm = sqrt(dot_chunked(vk, vk, n));
            for (int r = 0; r < n; ++r) vk[r] = vk[r] / nrm;
            R[k + k * K] = nrm;
            xi[k] = dot_chunked(res, vk, n);
        }
        /* truncation on the R diagonal (index stride = K, the loop value) */
        for (int i = 0; i < k; ++i)
            if (fabs(R[i + i * k]) < rel_tol * R[0]) { k = i; break; }
        const int full = k;
        /* error estimator */
        for (int i = 0; i < k; ++i) {
            iters += 1;
            if (xi[i] >= rho || xi[i] <= -rho) { k = i; break; }
            rho *= sin(acos(xi[i] / rho));
        }
        /* back-substitution; R indexed with stride full_krylov_dim exactly as
         * the reference does (GMRESSolver.cpp:331-337) */
        for (int i2 = k - 1; i2 > -1; --i2) {
            for (int jv = i2 + 1; jv < k; ++jv) xi[i2] -= R[i2 + jv * full] * xi[jv];
            xi[i2] /= R[i2 + i2 * full];
        }
        for (int i = 0; i < k; ++i) xi[i] *= rho0;
        /* gmres_update_result: coefficient 0 multiplies the residual, j >= 1
         * the basis vector j-1; coefficient 0 is applied even when k == 0 */
        for (int r = 0; r < n; ++r) {
            double v = x[r] + xi[0] * res[r];
            for (int jv = 1; jv < k; ++jv) v += xi[jv] * V[(size_t)(jv - 1) * n + r];
            x[r] = v;
        }
        st->prev_err = fabs(rho * rho0 / norm_rhs);
    }
    /* addInitialGuess */
    for (int r = 0; r < n; ++r) x[r] += x0[r];
    st->iters = iters;
    st->rho0 = rho0;
    free(res); free(x0); free(V); free(tmp);
}

/* ------------------------------------------------------------------------ */
/* kOmega::Solve (kOmega.cpp:31-73) with halveTimeStep / doubleTimeStep
 * (387-414).  The reference's "previous solution" copies act on solver
 * objects that are never created (kOmega.cpp:37-38, 395-396), so a halving
 * restores nothing; that is restated as is. */
/* A solve stopped by a NaN residual at its first convergence check: one
 * restart entered, no iteration, the field untouched (test hook). */
static void orc_fail_stats(orc_gmres_stats* st) {
    memset(st, 0, sizeof(*st));
    st->restarts = 1;
    st->nan = 1;
}

static void orc_halve(orc_komega_state* s, int* cur) {
    s->steps_per_lb *= 2;
    s->dt /= 2.0;
    *cur = 0;
    s->time_since_change = 0;
}

void orc_komega_solve(const orc_cfg* c, orc_komega_state* s,
                      const int16_t* map, const int32_t* IA, const int32_t* JA,
                      const int32_t* ind, double* K, double* O,
                      const double* nut, const double* wallD, const double* rho,
                      const double* ux, const double* uy, const double* Sxy,
                      const double* dX, double* Dk, double* Do, double* F1,
                      double* dkdo, double* kA, double* oA, double* kb,
                      double* ob) {
    const int n = c->nxf * c->ny;
    s->time_since_change++;
    if (s->time_since_change >= 20) {
        s->time_since_change = 0;
        if (s->steps_per_lb != 1) { s->steps_per_lb /= 2; s->dt *= 2.0; }
    }
    int cur = 0;
    while (cur < s->steps_per_lb) {
        orc_komega_diffusivities(c, map, K, O, nut, wallD, Dk, Do, F1, dkdo,
                                 rho, dX);
        orc_komega_coeffs(c, ind, K, O, nut, Dk, Do, F1, dkdo, Sxy, rho, ux,
                          uy, kA, oA, kb, ob, dX, wallD, map, s->dt);
        const int fail = s->fail_solves > 0 ? s->fail_mask : 0;
        if (s->fail_solves > 0) s->fail_solves--;
        if (fail & 1) orc_fail_stats(&s->last_o);
        else orc_gmres_solve(n, IA, JA, oA, ob, O, 10, s->max_iters, s->rel_tol,
                             s->abs_tol, &s->last_o);
        if (s->last_o.nan) orc_halve(s, &cur);
        if (fail & 2) orc_fail_stats(&s->last_k);
        else orc_gmres_solve(n, IA, JA, kA, kb, K, 10, s->max_iters, s->rel_tol,
                             s->abs_tol, &s->last_k);
        if (s->last_k.nan) orc_halve(s, &cur);
        /* A NaN that persists halves dt without end in the reference (the
         * state is not restored); stop at 2^20 sub-steps, as the product does. */
        if (s->steps_per_lb > (1 << 20)) break;
        cur++;
    }
}

/* ------------------------------------------------------------------------ */
/* Straight channel with half-way walls at y = 0.5 and y = nY - 1.5: the
 * geometry the reference builds from two straight wall polylines
 * (clVariablesLS.cpp:686-1000: iniFillMap0/iniFillMap, iniNodeBoundaryInfo0/
 * iniNodeBoundaryInfo, inidXArrays) and kOmega::iniWallD (kOmega.cpp:330-349). */
void orc_geom_straight(const orc_cfg* c, int16_t* map, double* dX,
                       double* wallD) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long D = (long)nxf * ny;
    const double yb = 0.5, yt = (double)ny - 1.5;
    for (long t = 0; t < D; ++t) { map[t] = 0; wallD[t] = 0.; }
    for (long t = 0; t < 4 * D; ++t) dX[t] = 0.;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nxf; ++i) {
            const long g = i + (long)nxf * j;
            if (i >= nx) { map[g] = (int16_t)(ORC_M0_FLUID | ORC_M_FLUID); continue; }
            const int solid = (j == 0 || j == ny - 1);
            map[g] = (int16_t)(solid ? (ORC_M0_SOLID | ORC_M_SOLID)
                                     : (ORC_M0_FLUID | ORC_M_FLUID));
        }
    for (int j = 1; j < ny - 1; ++j)
        for (int i = 0; i < nx; ++i) {
            const long g = i + (long)nxf * j;
            int t = (uint16_t)map[g];
            for (int q = 1; q < 9; ++q) {
                const int ii = (i + CX[q] + nx) % nx, jj = j + CY[q];
                const long gn = ii + (long)nxf * jj;
                if ((uint16_t)map[gn] & ORC_M_SOLID) {
                    t |= BOUND[q] | ORC_BOUNDARY0;
                    if (q < 5) {
                        t |= ORC_NESW_BOUNDARY0;
                        map[gn] = (int16_t)((uint16_t)map[gn] | ORC_SOLID_BOUNDARY | ORC_SOLID_BOUNDARY0);
                    }
                }
            }
            map[g] = (int16_t)t;
            dX[g] = 1.; dX[g + D] = 1.;
            dX[g + 2 * D] = (j == ny - 2) ? (yt - (double)j) : 1.;
            dX[g + 3 * D] = (j == 1) ? ((double)j - yb) : 1.;
            wallD[g] = dmin((double)j - yb, yt - (double)j);
        }
}

/* ------------------------------------------------------------------------ */
double orc_sum(const double* a, int64_t n) {
    double part[ORC_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) {
        const long s = (long)((cidx * (double)n) / ORC_CHUNKS);
        const long e = (long)(((cidx + 1) * (double)n) / ORC_CHUNKS);
        double acc = 0.;
        for (long t = s; t < e; ++t) acc += a[t];
        part[cidx] = acc;
    }
    double sum = 0.;
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) sum += part[cidx];
    return sum;
}

double orc_min(const double* a, int64_t n) {
    double m = a[0];
    for (int64_t t = 1; t < n; ++t) if (a[t] < m) m = a[t];
    return m;
}


/* TR_shear_1 (Kernels/trKernelsShear.cl:131-222): f_neq of populations 1..8
 * against the product-form equilibrium of the node's moments (calcLBDists),
 * dotted with the node's two coefficient rows and scaled by
 * (nu + nu_t) / (3 (nu + nu_t) + 1/2); tau = |.| / rho, signed by x. */
void orc_wall_shear_nodes(const orc_cfg* c, const double* FA, const double* rho,
                          const double* ux, const double* uy, const double* nut,
                          const int32_t* nodes, int n, const double* cfss, double* tau) {
    const long D = (long)c->nxf * c->ny;
    for (int i = 0; i < n; ++i) {
        const long g = nodes[i];
        double feq[9];
        orc_feq(rho[g], ux[g], uy[g], feq);
        double tx = 0.0, ty = 0.0;
        for (int q = 1; q < 9; ++q) {
            const double fneq = FA[g + q * D] - feq[q];
            tx += fneq * cfss[16L * i + q - 1];
            ty += fneq * cfss[16L * i + 8 + q - 1];
        }
        double visc = (nut ? nut[g] : 0.0) + c->mu;
        visc *= 1.0 / (3.0 * visc + 0.5);
        const double t = sqrt((tx * visc) * (tx * visc) + (ty * visc) * (ty * visc)) / rho[g];
        tau[i] = tx < 0.0 ? -t : t;
    }
}

/* TR_shear_2 (trKernelsShear.cl:300-316) */
void orc_wall_shear_links(const double* tau_nodes, const int32_t* sind, const double* w,
                          int nbl, double* out) {
    for (int b = 0; b < nbl; ++b) {
        double acc = 0.0;
        for (int a = 0; a < 4; ++a) {
            const int j = sind[4 * b + a];
            if (j >= 0) acc += w[4 * b + a] * tau_nodes[j];
        }
        out[b] = acc;
    }
}

/* ======================================================================== */
/* Thermal implicit finite differences (clVariablesFD::Solve,
 * clVariablesFD.h:343-358; Update_T_Coeffs_Implicit, tfdKernels.cl:122-279;
 * BiCGStabSolver::solve, BiCGStabSolver.cpp:628-723).                      */

/* CSR_Inds with flags (M0_SOLID, M0_FLUID, SOLID_BOUNDARY0) and no periodic
 * wrap (SparseMatrix.cpp:57-209, SparseMatrix.h:120-128; clVariablesFD.h:40):
 * rows of unfouled-wall boundary nodes hold only the diagonal, other wall
 * rows are empty, rows of the thermal domain (fluid and fouling layer) hold
 * S, W, C, E, N with the neighbours outside the lattice (x < 0, x >= nx)
 * left out. */
static int csr_th_neigh_ok(const orc_cfg* c, const int16_t* map, int i, int j) {
    if (i < 0 || i >= c->nx || j < 0 || j >= c->ny) return 0;
    const int t = (uint16_t)map[i + (long)c->nxf * j];
    return (t & (ORC_SOLID_BOUNDARY0 | ORC_M0_FLUID)) != 0;
}

int orc_csr_build_thermal(const orc_cfg* c, const int16_t* map, int32_t* IA,
                          int32_t* JA, int32_t* ind) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long n = (long)nxf * ny;
    enum { iC = 0, iE = 1, iW = 2, iN = 3, iS = 4 };
    int nnz = 0;
    if (IA) IA[0] = 0;
    if (ind) for (long t = 0; t < 5 * n; ++t) ind[t] = -1;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nxf; ++i) {
            const long g = i + (long)nxf * j;
            if (i < nx) {
                const int t = (uint16_t)map[g];
                if (t & ORC_M0_SOLID) {
                    if (t & ORC_SOLID_BOUNDARY0) {
                        if (JA) JA[nnz] = (int32_t)g;
                        if (ind) ind[g + n * iC] = nnz;
                        ++nnz;
                    }
                } else {
                    const long nb[5] = {g, g + 1, g - 1, g + nxf, g - nxf};
                    const int ok[5] = {1, csr_th_neigh_ok(c, map, i + 1, j),
                                       csr_th_neigh_ok(c, map, i - 1, j),
                                       csr_th_neigh_ok(c, map, i, j + 1),
                                       csr_th_neigh_ok(c, map, i, j - 1)};
                    const int order[5] = {iS, iW, iC, iE, iN};
                    for (int k = 0; k < 5; ++k) {
                        const int d = order[k];
                        if (!ok[d]) continue;
                        if (JA) JA[nnz] = (int32_t)nb[d];
                        if (ind) ind[g + n * d] = nnz;
                        ++nnz;
                    }
                }
            }
            if (IA) IA[g + 1] = nnz;
        }
    return nnz;
}

void orc_csr_fill_solid_boundary_thermal(const orc_cfg* c, const int16_t* map,
                                         const int32_t* ind, double* A) {
    for (int j = 0; j < c->ny; ++j)
        for (int i = 0; i < c->nx; ++i) {
            const long g = i + (long)c->nxf * j;
            const int t = (uint16_t)map[g];
            if ((t & ORC_M0_SOLID) && (t & ORC_SOLID_BOUNDARY0)) A[ind[g]] = 1.;
        }
}

/* Update_T_Coeffs_Implicit (tfdKernels.cl:122-279): backward-Euler rows of
 * the advection-diffusion equation of T with non-uniform 3-point differences
 * from the link fractions dX0 (floored at 0.1), the advecting flux
 * J = u - grad(nu_t)/Pr_t, diffusivity alpha (+ nu_t/Pr_t), fixed inlet
 * temperature on x = 0 (its W term moved to the right-hand side) and a
 * zero-gradient outlet on x = nx-1 (its E term added to the diagonal); every
 * row is divided by its diagonal.  Rows of unfouled-wall nodes are left as
 * they are. */
void orc_thermal_coeffs(const orc_cfg* c, const orc_thermal_cfg* th, const int32_t* ind,
                        const int16_t* map, const double* dX0, double* A, double* b,
                        const double* T, const double* ux, const double* uy,
                        const double* nut, double dt) {
    const int nx = c->nx, nxf = c->nxf, ny = c->ny;
    const long D = (long)nxf * ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const long g = i + (long)nxf * j;
            const int t = (uint16_t)map[g];
            if (t & ORC_M0_SOLID) continue;
            const double dxe = dmax(dX0[g], 0.1), dxw = dmax(dX0[g + D], 0.1);
            const double dxc = dmax(dxe + dxw, 0.1);
            const double dyn = dmax(dX0[g + 2 * D], 0.1), dys = dmax(dX0[g + 3 * D], 0.1);
            const double dyc = dmax(dyn + dys, 0.1);
            double dXe = dxw / (dxe * dxc), dXw = -dxe / (dxw * dxc), dXc = (dxe - dxw) / (dxe * dxw);
            double dYn = dys / (dyn * dyc), dYs = -dyn / (dys * dyc), dYc = (dyn - dys) / (dyn * dys);
            const double dX2e = 2. / (dxe * dxc), dX2w = 2. / (dxw * dxc), dX2c = -2. / (dxe * dxw);
            const double dY2n = 2. / (dyn * dyc), dY2s = 2. / (dys * dyc), dY2c = -2. / (dyn * dys);
            if (fabs(dXc) > 10.) { dXe = 1.0 / dxc; dXw = -1.0 / dxc; dXc = 0.0; }
            if (fabs(dYn) > 10.) { dYn = 1.0 / dyc; dYs = -1.0 / dyc; dYc = 0.0; }
            double alpha = (t & ORC_M_SOLID) ? th->alpha_foul : th->alpha_fluid;
            const double nu_c = nut ? nut[g] : 0.0;
            const double alphat = nu_c * th->pr_turb_inv;
            const long gw = (i > 0 ? -1 : nx - 1) + g;
            const long ge = (i < nx - 1 ? 1 : 1 - nxf) + g;
            const double nu_e = nut ? nut[ge] : 0.0, nu_w = nut ? nut[gw] : 0.0;
            const double nu_n = nut ? nut[g + nxf] : 0.0, nu_s = nut ? nut[g - nxf] : 0.0;
            const double Jx = ux[g] - (th->pr_turb_inv * (dXe * nu_e + dXw * nu_w + dXc * alphat));
            const double Jy = uy[g] - (th->pr_turb_inv * (dYn * nu_n + dYs * nu_s + dYc * alphat));
            alpha += alphat;
            double Tsrc = dmin(dmax(0.0, T[g]), th->t_in);
            double Cc = 1. + dt * (Jx * dXc + Jy * dYc - alpha * (dX2c + dY2c));
            const double Sc = dt * (Jy * dYs - alpha * dY2s);
            const double Wc = dt * (Jx * dXw - alpha * dX2w);
            if (i == 0) Tsrc -= th->t_in * Wc;
            const double Ec = dt * (Jx * dXe - alpha * dX2e);
            if (i == nx - 1) Cc += Ec;
            Cc = 1. / Cc;
            A[ind[g + 4 * D]] = Sc * Cc;
            if (i > 0) A[ind[g + 2 * D]] = Wc * Cc;
            if (i < nx - 1) A[ind[g + D]] = Ec * Cc;
            A[ind[g]] = 1.;
            A[ind[g + 3 * D]] = dt * (Jy * dYn - alpha * dY2n) * Cc;
            b[g] = Tsrc * Cc;
        }
}

static double sum_abs_chunked(const double* a, long n) {
    double part[ORC_CHUNKS];
#pragma omp parallel for schedule(static)
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) {
        const long s = (long)((cidx * (double)n) / ORC_CHUNKS);
        const long e = (long)(((cidx + 1) * (double)n) / ORC_CHUNKS);
        double acc = 0.;
        for (long t = s; t < e; ++t) acc += fabs(a[t]);
        part[cidx] = acc;
    }
    double sum = 0.;
    for (int cidx = 0; cidx < ORC_CHUNKS; ++cidx) sum += part[cidx];
    return sum;
}

/* reduceAndCheckConvergence (BiCGStabSolver.cpp:509-545): the residual is
 * the L1 norm of r over the L1 norm of b ("Norm" reduction,
 * BiCGStabGenerator.cpp:259-262). */
static int bicg_check(orc_bicgstab_stats* st, const double* r, long n, double normb,
                      int first, int iter, double* avg, double rel_tol, double abs_tol,
                      int reset_flag) {
    const double res = sum_abs_chunked(r, n) / normb;
    st->checks++;
    st->residual = res;
    if (first) st->initial_residual = res;
    if (reset_flag && (isnan(res) || (iter > 1 && res > 10. * *avg))) {
        st->reset = 1;
        return 1;
    }
    if (res <= rel_tol || res <= abs_tol * st->initial_residual) {
        st->conv = 1;
        return 1;
    }
    *avg = res;
    return 0;
}

/* BiCGStabSolver::solve (BiCGStabSolver.cpp:628-723) as the reference
 * enqueues it.  The scalars start at 1 on every call (scalarBuf.FillBuffer);
 * omega is never reduced (the omegaDotSqr list is built but not run), so
 * every "omega" update uses 1; step f9 recomputes alpha from the same
 * vectors.  b is overwritten with the residual; x holds the initial guess on
 * entry.  With reset_flag, a NaN residual or one that grew tenfold since the
 * previous check (after the second iteration) stops the solve with
 * st->reset = 1 (the resetTimeFunc path). */
void orc_bicgstab_solve(int n, const int32_t* IA, const int32_t* JA, const double* A,
                        double* b, double* x, int max_iters, double rel_tol, double abs_tol,
                        int reset_flag, orc_bicgstab_stats* st) {
    memset(st, 0, sizeof(*st));
    double* r0 = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* v = (double*)malloc(sizeof(double) * n);
    double* t = (double*)malloc(sizeof(double) * n);
    double rho = 1., alpha = 1., omega = 1., beta = 1., avg = 0.;
    const double normb = sum_abs_chunked(b, n);
    int iter = 0;
    if (normb <= 1.0e-16) {
        memcpy(x, b, sizeof(double) * n);
        st->conv = 1;
        goto done;
    }
    spmv(n, IA, JA, A, x, t);
    for (int k = 0; k < n; ++k) b[k] -= t[k];
    memcpy(r0, b, sizeof(double) * n);
    memcpy(p, b, sizeof(double) * n);
    rho = dot_chunked(b, b, n);
    int first = 1;
    while (iter < max_iters) {
        if (iter > 0) {
            const double rho_new = dot_chunked(b, r0, n);
            beta = (rho_new / rho) * (alpha / omega);
            rho = rho_new;
            for (int k = 0; k < n; ++k) p[k] = b[k] + beta * (p[k] - omega * v[k]);
        }
        spmv(n, IA, JA, A, p, v);
        alpha = rho / dot_chunked(v, r0, n);
        for (int k = 0; k < n; ++k) {
            x[k] += alpha * p[k];
            b[k] -= alpha * v[k];
        }
        if (bicg_check(st, b, n, normb, first, iter, &avg, rel_tol, abs_tol, reset_flag)) break;
        first = 0;
        spmv(n, IA, JA, A, b, t);
        alpha = rho / dot_chunked(v, r0, n);
        for (int k = 0; k < n; ++k) {
            x[k] += omega * b[k];
            b[k] -= omega * t[k];
        }
        if (bicg_check(st, b, n, normb, first, iter, &avg, rel_tol, abs_tol, reset_flag)) break;
        iter++;
    }
done:
    st->iters = iter;
    free(r0); free(p); free(v); free(t);
}

/* clVariablesFD::Solve (clVariablesFD.h:343-358) with halveTimeStep /
 * doubleTimeStep (clVariablesFD.cpp:202-228): T is saved before the
 * sub-steps; a reset restores it, doubles the sub-step count and halves dt,
 * and the sub-step loop continues from its counter's restart. */
void orc_thermal_solve(const orc_cfg* c, const orc_thermal_cfg* th, orc_thermal_state* s,
                       const int16_t* map, const int32_t* IA, const int32_t* JA,
                       const int32_t* ind, const double* dX0, double* T, double* Tprev,
                       const double* ux, const double* uy, const double* nut, double* A,
                       double* b) {
    const int n = c->nxf * c->ny;
    s->time_since_change++;
    if (s->time_since_change >= 20) {
        s->time_since_change = 0;
        if (s->steps_per_lb != 1) { s->steps_per_lb /= 2; s->dt *= 2.0; }
    }
    memcpy(Tprev, T, sizeof(double) * n);
    int cur = 0;
    s->solves = 0;
    s->resets = 0;
    while (cur < s->steps_per_lb) {
        orc_thermal_coeffs(c, th, ind, map, dX0, A, b, T, ux, uy, nut, s->dt);
        orc_bicgstab_solve(n, IA, JA, A, b, T, s->max_iters, s->rel_tol, s->abs_tol, 1, &s->last);
        s->solves++;
        if (s->last.reset) {
            s->steps_per_lb *= 2;
            s->dt /= 2.0;
            memcpy(T, Tprev, sizeof(double) * n);
            cur = 0;
            s->time_since_change = 0;
            s->resets++;
        }
        if (s->steps_per_lb > (1 << 20)) break;
        cur++;
    }
}
