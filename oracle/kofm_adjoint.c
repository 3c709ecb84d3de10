/* kofm_adjoint.c - FP64 CPU restatement of the discrete adjoint of the
 * laminar D2Q9 step (TEST INFRASTRUCTURE ONLY: the checker of the device
 * adjoint; the product never links it).
 *
 * The reference has no adjoint.  What is differentiated is the reference's
 * laminar step as the oracle restates it (kofm_oracle.c): collide
 * (LB_collision_SRT_Fluid, lbKernels.cl:175-335: BGK with exact-difference
 * forcing), push stream with half-way bounce-back, then lbIBB
 * (lbKernels.cl:640-668, Bouzidi linear interpolation with wall fraction q).
 *
 * Notation: f*^n = post-collision populations produced from FA^n (stored at
 * the producing node, f*_i(x)); FA^{n+1} = IBB(push(f*^n)).  A run of T steps
 * starts from FA^0, forms f*^0 = C(FA^0) and visits FA^1 .. FA^T;
 * J = sum_{n=1..T} j(FA^n) with
 *   j(F) = (rho_in - rho_out) / 3 + sum_s tau_s(F)
 * rho_in / rho_out the mean density over the fluid nodes of columns 0 and
 * nx-1, tau_s the wall shear of TR_shear_1 (trKernelsShear.cl:175-222) at
 * shear node s computed from F and F's own moments (reported u_x = u_x +
 * fterm/2, laminar viscosity).  The adjoint recursion is
 *   lambda^T = dj/dFA^T,
 *   nu^n = (d FA^{n+1} / d f*^n)^T lambda^{n+1},
 *   lambda^n = dj/dFA^n + (d f*^n / d FA^n)^T nu^n     (n >= 1),
 *   dJ/dq_l += lambda^{n+1}[link l] * d FA^{n+1}[link l] / dq_l,
 * and dJ/dFA^0 = (d f*^0 / d FA^0)^T nu^0.
 */
#include "kofm_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const int ACX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
static const int ACY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
static const int AREV[9] = {0, 2, 1, 4, 3, 6, 5, 8, 7};
static const int ABOUND[9] = {0, 0x100, 0x200, 0x400, 0x800, 0x1000, 0x2000, 0x4000, 0x8000};

static inline double phi(int c, double u) { return c == 0 ? 2. / 3. - u * u : 0.5 * (1. / 3. + c * u + u * u); }
static inline double dphi(int c, double u) { return c == 0 ? -2. * u : 0.5 * (c + 2. * u); }

/* collide of one node (the laminar branch of orc_collide_push) */
static void collide_node(const orc_cfg* c, const double* f, double* out) {
    double rho = 0.;
    for (int q = 0; q < 9; ++q) rho += f[q];
    const double inv = 1. / rho;
    const double ux = inv * (f[1] - f[2] + f[5] - f[6] + f[7] - f[8]);
    const double uy = inv * (f[3] - f[4] + f[5] - f[6] - f[7] + f[8]);
    const double w = c->tau0;
    double feq[9], feqF[9];
    orc_feq(rho, ux, uy, feq);
    orc_feq(rho, ux + c->fterm, uy, feqF);
    for (int q = 0; q < 9; ++q) out[q] = f[q] - w * (f[q] - feq[q]) - feq[q] + feqF[q];
}

/* (d collide / d f)^T nu at one node, added to lam */
static void collide_T_node(const orc_cfg* c, const double* f, const double* nu, double* lam) {
    double rho = 0.;
    for (int q = 0; q < 9; ++q) rho += f[q];
    const double inv = 1. / rho;
    const double ux = inv * (f[1] - f[2] + f[5] - f[6] + f[7] - f[8]);
    const double uy = inv * (f[3] - f[4] + f[5] - f[6] - f[7] + f[8]);
    const double w = c->tau0, uf = ux + c->fterm;
    /* f*_i = (1-w) f_i + (w-1) feq_i(rho,u) + feq_i(rho,u+F);
     * d feq_i / d f_j = PhiPhi_i + rho dPhi_i/du . (c_j - u) / rho */
    double A = 0., Bx = 0., By = 0.;
    for (int i = 0; i < 9; ++i) {
        const double p0x = phi(ACX[i], ux), p0y = phi(ACY[i], uy);
        const double pFx = phi(ACX[i], uf);
        A += nu[i] * ((w - 1.) * p0x * p0y + pFx * p0y);
        Bx += nu[i] * ((w - 1.) * dphi(ACX[i], ux) * p0y + dphi(ACX[i], uf) * p0y);
        By += nu[i] * ((w - 1.) * p0x + pFx) * dphi(ACY[i], uy);
    }
    for (int j = 0; j < 9; ++j)
        lam[j] += (1. - w) * nu[j] + A + Bx * (ACX[j] - ux) + By * (ACY[j] - uy);
}

void orc_adj_collide(const orc_cfg* c, const int16_t* map, const double* FA, double* fstar) {
    const long D = (long)c->nxf * c->ny;
    memset(fstar, 0, sizeof(double) * 9 * D);
    for (int y = 0; y < c->ny; ++y)
        for (int x = 0; x < c->nx; ++x) {
            const long g = x + (long)c->nxf * y;
            if ((uint16_t)map[g] & ORC_M_SOLID) continue;
            double f[9], o[9];
            for (int q = 0; q < 9; ++q) f[q] = FA[g + q * D];
            collide_node(c, f, o);
            for (int q = 0; q < 9; ++q) fstar[g + q * D] = o[q];
        }
}

/* push with half-way bounce-back (orc_collide_push's stream part) */
static void push(const orc_cfg* c, const int16_t* map, const double* fs, double* FB) {
    const int nx = c->nx, nxf = c->nxf;
    const long D = (long)nxf * c->ny;
    memset(FB, 0, sizeof(double) * 9 * D);
    for (int y = 0; y < c->ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const long g = x + (long)nxf * y;
            const int t = (uint16_t)map[g];
            if (t & ORC_M_SOLID) continue;
            FB[g] = fs[g];
            for (int q = 1; q < 9; ++q) {
                if (t & ABOUND[q]) {
                    FB[g + D * AREV[q]] = fs[g + D * q];
                } else {
                    const int xd = ((x + ACX[q]) % nx + nx) % nx;
                    FB[xd + (long)nxf * (y + ACY[q]) + D * q] = fs[g + D * q];
                }
            }
        }
}

void orc_adj_stream(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                    int nibb, const double* fstar, double* FA) {
    push(c, map, fstar, FA);
    orc_ibb(c, ibb, q, FA, nibb);
}

/* nu = (d FA / d f*)^T lam, and dq += lam . d FA / d q */
void orc_adj_stream_T(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                      int nibb, const double* lam, const double* fstar, double* nu, double* dq) {
    const int nx = c->nx, nxf = c->nxf;
    const long D = (long)nxf * c->ny;
    double* FB = (double*)malloc(sizeof(double) * 9 * D);
    double* lc = (double*)malloc(sizeof(double) * 9 * D);
    push(c, map, fstar, FB);
    memcpy(lc, lam, sizeof(double) * 9 * D);
    /* the IBB updates read pushed values only (no link reads another link's
     * result), so every derivative uses FB as pushed */
    for (int l = nibb - 1; l >= 0; --l) {
        const long loc = ibb[l];
        const int dir = (int)(loc / D);
        const long node = loc - (long)dir * D;
        const long rev = node + D * AREV[dir];
        const double twoQ = 2. * q[l];
        const double lr = lc[rev];
        if (twoQ <= 1.0) {
            dq[l] += lr * 2. * (FB[rev] - FB[loc]);
            lc[loc] += (1. - twoQ) * lr;
            lc[rev] = twoQ * lr;
        } else {
            const long up = node - ACX[dir] - (long)ACY[dir] * nxf;
            const long revNeigh = up + D * AREV[dir];
            dq[l] += lr * (FB[revNeigh] - FB[rev]) / (2. * q[l] * q[l]);
            lc[revNeigh] += (twoQ - 1.) / twoQ * lr;
            lc[rev] = lr / twoQ;
        }
    }
    memset(nu, 0, sizeof(double) * 9 * D);
    for (int y = 0; y < c->ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const long g = x + (long)nxf * y;
            const int t = (uint16_t)map[g];
            if (t & ORC_M_SOLID) continue;
            nu[g] = lc[g];
            for (int qq = 1; qq < 9; ++qq) {
                if (t & ABOUND[qq]) {
                    nu[g + D * qq] = lc[g + D * AREV[qq]];
                } else {
                    const int xd = ((x + ACX[qq]) % nx + nx) % nx;
                    nu[g + D * qq] = lc[xd + (long)nxf * (y + ACY[qq]) + D * qq];
                }
            }
        }
    free(FB);
    free(lc);
}

/* fluid node counts of columns 0 and nx-1 */
static void edge_counts(const orc_cfg* c, const int16_t* map, int* n0, int* n1) {
    *n0 = *n1 = 0;
    for (int y = 0; y < c->ny; ++y) {
        if (!((uint16_t)map[(long)c->nxf * y] & ORC_M_SOLID)) ++*n0;
        if (!((uint16_t)map[c->nx - 1 + (long)c->nxf * y] & ORC_M_SOLID)) ++*n1;
    }
}

/* tau of TR_shear_1 from F and F's own moments; grad (nullable) += d tau / d F */
static double shear_node(const orc_cfg* c, const double* F, const double* cf, double* grad) {
    double rho = 0.;
    for (int q = 0; q < 9; ++q) rho += F[q];
    const double inv = 1. / rho;
    const double ux = inv * (F[1] - F[2] + F[5] - F[6] + F[7] - F[8]);
    const double uy = inv * (F[3] - F[4] + F[5] - F[6] - F[7] + F[8]);
    const double ur = ux + 0.5 * c->fterm;
    double visc = c->mu;
    visc *= 1.0 / (3.0 * visc + 0.5);
    double tx = 0., ty = 0., Ax = 0., Ay = 0., Bxx = 0., Bxy = 0., Byx = 0., Byy = 0.;
    for (int q = 1; q < 9; ++q) {
        const double px = phi(ACX[q], ur), py = phi(ACY[q], uy);
        const double fneq = F[q] - rho * px * py;
        tx += fneq * cf[q - 1];
        ty += fneq * cf[8 + q - 1];
        Ax += cf[q - 1] * px * py;
        Ay += cf[8 + q - 1] * px * py;
        Bxx += cf[q - 1] * dphi(ACX[q], ur) * py;
        Bxy += cf[q - 1] * px * dphi(ACY[q], uy);
        Byx += cf[8 + q - 1] * dphi(ACX[q], ur) * py;
        Byy += cf[8 + q - 1] * px * dphi(ACY[q], uy);
    }
    const double T = sqrt(tx * tx + ty * ty);
    const double sg = tx < 0. ? -1. : 1.;
    const double tau = sg * visc * T / rho;
    if (grad && T > 0.) {
        for (int j = 0; j < 9; ++j) {
            const double dux = (ACX[j] - ux), duy = (ACY[j] - uy);  /* rho d u / d F_j */
            const double dtx = (j > 0 ? cf[j - 1] : 0.) - Ax - Bxx * dux - Bxy * duy;
            const double dty = (j > 0 ? cf[8 + j - 1] : 0.) - Ay - Byx * dux - Byy * duy;
            grad[j] += sg * visc * ((tx * dtx + ty * dty) / (T * rho) - T / (rho * rho));
        }
    }
    return tau;
}

double orc_adj_j(const orc_cfg* c, const int16_t* map, const double* FA, const int32_t* snodes,
                 const double* cfss, int nshear, double* grad) {
    const long D = (long)c->nxf * c->ny;
    int n0, n1;
    edge_counts(c, map, &n0, &n1);
    double r0 = 0., r1 = 0.;
    for (int y = 0; y < c->ny; ++y) {
        const long g0 = (long)c->nxf * y, g1 = c->nx - 1 + (long)c->nxf * y;
        if (!((uint16_t)map[g0] & ORC_M_SOLID))
            for (int q = 0; q < 9; ++q) {
                r0 += FA[g0 + q * D];
                if (grad) grad[g0 + q * D] += 1. / (3. * n0);
            }
        if (!((uint16_t)map[g1] & ORC_M_SOLID))
            for (int q = 0; q < 9; ++q) {
                r1 += FA[g1 + q * D];
                if (grad) grad[g1 + q * D] -= 1. / (3. * n1);
            }
    }
    double j = (r0 / n0 - r1 / n1) / 3.;
    for (int s = 0; s < nshear; ++s) {
        const long g = snodes[s];
        double F[9], gr[9] = {0};
        for (int q = 0; q < 9; ++q) F[q] = FA[g + q * D];
        j += shear_node(c, F, cfss + 16L * s, grad ? gr : NULL);
        if (grad)
            for (int q = 0; q < 9; ++q) grad[g + q * D] += gr[q];
    }
    return j;
}

/* A whole run: J and its gradients with respect to the IBB wall fractions
 * (dq, nibb entries) and to FA^0 (dF0, nullable).  Every state is kept
 * (small lattices only). */
double orc_adj_run(const orc_cfg* c, const int16_t* map, const int32_t* ibb, const double* q,
                   int nibb, const double* FA0, int T, const int32_t* snodes, const double* cfss,
                   int nshear, double* dq, double* dF0) {
    const long D = (long)c->nxf * c->ny;
    const size_t S = sizeof(double) * 9 * D;
    double* fs = (double*)malloc(S * (size_t)T);   /* f*^0 .. f*^{T-1} */
    double* fa = (double*)malloc(S * (size_t)(T + 1)); /* FA^0 .. FA^T */
    double* lam = (double*)malloc(S);
    double* nu = (double*)malloc(S);
    memcpy(fa, FA0, S);
    double J = 0.;
    for (int n = 0; n < T; ++n) {
        orc_adj_collide(c, map, fa + (size_t)n * 9 * D, fs + (size_t)n * 9 * D);
        orc_adj_stream(c, map, ibb, q, nibb, fs + (size_t)n * 9 * D, fa + (size_t)(n + 1) * 9 * D);
        J += orc_adj_j(c, map, fa + (size_t)(n + 1) * 9 * D, snodes, cfss, nshear, NULL);
    }
    if (dq) memset(dq, 0, sizeof(double) * (size_t)nibb);
    memset(lam, 0, S);
    orc_adj_j(c, map, fa + (size_t)T * 9 * D, snodes, cfss, nshear, lam);
    double* dqw = dq ? dq : (double*)calloc((size_t)(nibb > 0 ? nibb : 1), sizeof(double));
    for (int n = T - 1; n >= 0; --n) {
        orc_adj_stream_T(c, map, ibb, q, nibb, lam, fs + (size_t)n * 9 * D, nu, dqw);
        memset(lam, 0, S);
        const double* F = fa + (size_t)n * 9 * D;
        if (n >= 1) orc_adj_j(c, map, F, snodes, cfss, nshear, lam);
        if (n >= 1 || dF0) {
            for (int y = 0; y < c->ny; ++y)
                for (int x = 0; x < c->nx; ++x) {
                    const long g = x + (long)c->nxf * y;
                    if ((uint16_t)map[g] & ORC_M_SOLID) continue;
                    double f[9], v[9], l[9];
                    for (int k = 0; k < 9; ++k) { f[k] = F[g + k * D]; v[k] = nu[g + k * D]; l[k] = 0.; }
                    collide_T_node(c, f, v, l);
                    for (int k = 0; k < 9; ++k) lam[g + k * D] += l[k];
                }
        }
    }
    if (dF0) memcpy(dF0, lam, S);
    if (!dq) free(dqw);
    free(fs); free(fa); free(lam); free(nu);
    return J;
}
