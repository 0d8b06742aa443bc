/*
 * kumo_oracle.c: CPU restatement of chem-kumo's grid-block evaluator.
 * TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline); see kumo_oracle.h.
 *
 * Compiled with -ffp-contract=off so that every product and sum is rounded as
 * written, in the order of the reference expressions (an x86-64 build of the
 * reference without -march uses no fused multiply-add either).
 */
#include "kumo_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KO_PI 3.141592653589793238462643383279502884

static void set_err(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) {
        strncpy(err, msg, (size_t)errlen - 1);
        err[errlen - 1] = '\0';
    }
}

/* ------------------------------------------------------------------ */
/* Basis preparation                                                   */
/* ------------------------------------------------------------------ */

typedef struct {
    double origin[3];
    int l, nprim, ncart, count, offset, pure;
    double* exps;    /* nprim */
    double* weights; /* ncart x nprim, row-major [k * nprim + p] */
    int (*powers)[3];
    double* transform; /* count x ncart row-major, NULL when not pure */
    double cutoff_r2;
} ko_block;

struct ko_basis {
    int nblocks, nao, max_l, max_prim, max_cart;
    ko_block* blocks;
};

/* src/basis_evaluator.cpp:15-22 */
static double factorial(int n) {
    double v = 1.0;
    for (long long i = 2; i <= n; ++i) v *= (double)i;
    return v;
}

/* src/basis_math.cpp:9-15 */
static double double_factorial_odd(int n) {
    if (n <= 0) return 1.0;
    double v = 1.0;
    for (int i = n; i >= 1; i -= 2) v *= (double)i;
    return v;
}

/* src/basis_math.cpp:17-25 */
double ko_primitive_norm(double alpha, int px, int py, int pz) {
    const int l = px + py + pz;
    const double radial = pow(2.0 * alpha / KO_PI, 0.75);
    const double angular = sqrt(pow(4.0 * alpha, (double)l) /
                                (double_factorial_odd(2 * px - 1) * double_factorial_odd(2 * py - 1) *
                                 double_factorial_odd(2 * pz - 1)));
    return radial * angular;
}

/* src/basis_evaluator.cpp:135-152 */
static int cartesian_order(int l, int (*out)[3]) {
    static const int d[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    static const int f[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {1, 2, 0}, {2, 1, 0},
                                 {2, 0, 1}, {1, 0, 2}, {0, 1, 2}, {0, 2, 1}, {1, 1, 1}};
    int n = 0;
    if (l == 0) {
        out[0][0] = out[0][1] = out[0][2] = 0;
        return 1;
    }
    if (l == 1) {
        for (int a = 0; a < 3; ++a) {
            out[a][0] = out[a][1] = out[a][2] = 0;
            out[a][a] = 1;
        }
        return 3;
    }
    if (l == 2) {
        memcpy(out, d, sizeof d);
        return 6;
    }
    if (l == 3) {
        memcpy(out, f, sizeof f);
        return 10;
    }
    for (int lx = 0; lx <= l; ++lx)
        for (int ly = 0; ly <= l - lx; ++ly) {
            out[n][0] = lx;
            out[n][1] = ly;
            out[n][2] = l - lx - ly;
            ++n;
        }
    return n;
}

/* src/basis_evaluator.cpp:49-83 (Schlegel and Frisch 1995) */
static double cartesian_to_pure_coefficient(int l, int m, int lx, int ly) {
    const int lz = l - lx - ly;
    const int ma = abs(m);
    if (ma > l || lz < 0) return 0.0;
    const double a = sqrt(factorial(2 * lx) * factorial(2 * ly) * factorial(2 * lz) * factorial(l) /
                          (factorial(2 * l) * factorial(lx) * factorial(ly) * factorial(lz)));
    const double b = sqrt(factorial(l - ma) / factorial(l + ma)) / (pow(2.0, l) * factorial(l));
    const int ilim = (l - ma) / 2;
    const int j = (l - ma - lz) / 2;
    double g = 0.0;
    if (2 * j != l - ma - lz) return 0.0;
    for (int i = 0; i <= ilim; ++i) {
        if (j < 0 || j > i) continue;
        const double c = factorial(l) / (factorial(i) * factorial(l - i)) * factorial(2 * l - 2 * i) *
                         pow(-1.0, i) / factorial(l - ma - 2 * i) * factorial(i) /
                         (factorial(j) * factorial(i - j));
        for (int k = 0; k <= j; ++k) {
            if (lx - 2 * k < 0 || lx - 2 * k > ma) continue;
            const double d = factorial(j) / (factorial(k) * factorial(j - k)) * factorial(ma) /
                             (factorial(lx - 2 * k) * factorial(ma + 2 * k - lx));
            double e = 0.0;
            const int k_minus_lx2 = k - lx / 2;
            if (m == 0 && (lx % 2) == 0) e = pow(-1.0, k_minus_lx2);
            const int kt = (2 * k + ma - lx) / 2;
            if (m > 0 && (abs(ma - lx) % 2) == 0) e = sqrt(2.0) * pow(-1.0, kt);
            if (m < 0 && (abs(ma - lx) % 2) == 1) e = sqrt(2.0) * pow(-1.0, kt);
            g += c * d * e;
        }
    }
    return a * b * g;
}

/* src/basis_evaluator.cpp:157-175; out column-major (2l+1) x ncart */
void ko_pure_transform(int l, double* out) {
    int pw[64][3];
    const int nc = cartesian_order(l, pw);
    const int rows = 2 * l + 1;
    for (int g = 0; g < nc; ++g) {
        out[g * rows + 0] = cartesian_to_pure_coefficient(l, 0, pw[g][0], pw[g][1]);
        for (int m = 1; m <= l; ++m) {
            out[g * rows + 2 * m - 1] = cartesian_to_pure_coefficient(l, m, pw[g][0], pw[g][1]);
            out[g * rows + 2 * m] = cartesian_to_pure_coefficient(l, -m, pw[g][0], pw[g][1]);
        }
    }
}

/* src/basis_evaluator.cpp:98-127 */
static double shell_cutoff_radius(const ko_block* blk, double transform_norm, double cutoff) {
    const int l = blk->l;
    double coefficient[64];
    double start = 1.0;
    for (int p = 0; p < blk->nprim; ++p) {
        const double a = blk->exps[p];
        double weight = 0.0;
        for (int k = 0; k < blk->ncart; ++k) {
            const double w = fabs(blk->weights[k * blk->nprim + p]);
            if (k == 0 || w > weight) weight = w;
        }
        coefficient[p] =
            transform_norm * weight * (1.0 + l + l * l + 2.0 * a * (2.0 * l + 2.0) + 4.0 * a * a);
        const double s = sqrt((l + 2.0) / (2.0 * a));
        if (s > start) start = s;
    }
#define KO_BOUND(r, out)                                                                         \
    do {                                                                                         \
        double sum_ = 0.0;                                                                       \
        for (int p_ = 0; p_ < blk->nprim; ++p_)                                                  \
            sum_ += coefficient[p_] * pow((r), (double)(l + 2)) * exp(-blk->exps[p_] * (r) * (r)); \
        (out) = sum_;                                                                            \
    } while (0)
    double bound;
    KO_BOUND(start, bound);
    if (bound <= cutoff) return start;
    double low = start, high = 2.0 * start;
    for (;;) {
        KO_BOUND(high, bound);
        if (!(bound > cutoff)) break;
        high *= 2.0;
    }
    for (int it = 0; it < 60; ++it) {
        const double middle = 0.5 * (low + high);
        KO_BOUND(middle, bound);
        if (bound > cutoff)
            low = middle;
        else
            high = middle;
    }
#undef KO_BOUND
    return high;
}

static void add_block(ko_basis* b, const double* origin, int l, int nprim, const double* exps,
                      const double* coefs, int pure, int* offset) {
    ko_block* blk = &b->blocks[b->nblocks++];
    memset(blk, 0, sizeof *blk);
    memcpy(blk->origin, origin, sizeof blk->origin);
    blk->l = l;
    blk->nprim = nprim;
    blk->exps = (double*)malloc(sizeof(double) * (size_t)nprim);
    memcpy(blk->exps, exps, sizeof(double) * (size_t)nprim);
    int pw[128][3];
    blk->ncart = cartesian_order(l, pw);
    blk->powers = malloc(sizeof(int[3]) * (size_t)blk->ncart);
    memcpy(blk->powers, pw, sizeof(int[3]) * (size_t)blk->ncart);
    blk->weights = (double*)malloc(sizeof(double) * (size_t)(blk->ncart * nprim));
    /* src/basis_math.cpp:41-45 */
    for (int k = 0; k < blk->ncart; ++k)
        for (int p = 0; p < nprim; ++p)
            blk->weights[k * nprim + p] =
                coefs[p] * ko_primitive_norm(exps[p], pw[k][0], pw[k][1], pw[k][2]);
    blk->pure = pure && l >= 2;
    double transform_norm = 1.0;
    if (blk->pure) {
        const int rows = 2 * l + 1;
        double* cm = (double*)malloc(sizeof(double) * (size_t)(rows * blk->ncart));
        ko_pure_transform(l, cm);
        blk->transform = (double*)malloc(sizeof(double) * (size_t)(rows * blk->ncart));
        for (int m = 0; m < rows; ++m)
            for (int k = 0; k < blk->ncart; ++k) blk->transform[m * blk->ncart + k] = cm[k * rows + m];
        free(cm);
        blk->count = rows;
        /* largest absolute row sum, src/basis_evaluator.cpp:190-192 */
        transform_norm = 0.0;
        for (int m = 0; m < rows; ++m) {
            double s = fabs(blk->transform[m * blk->ncart]);
            for (int k = 1; k < blk->ncart; ++k) s += fabs(blk->transform[m * blk->ncart + k]);
            if (m == 0 || s > transform_norm) transform_norm = s;
        }
    } else {
        blk->count = blk->ncart;
    }
    blk->offset = *offset;
    *offset += blk->count;
    const double r = shell_cutoff_radius(blk, transform_norm, 1e-14);
    blk->cutoff_r2 = r * r;
    if (l > b->max_l) b->max_l = l;
    if (nprim > b->max_prim) b->max_prim = nprim;
    if (blk->ncart > b->max_cart) b->max_cart = blk->ncart;
}

ko_basis* ko_basis_create(int nshell, const int* shell_types, const int* nprim, const double* exps,
                          const double* coefs, const double* p_coefs, const double* shell_xyz,
                          int declared_nbasis, char* err, int errlen) {
    ko_basis* b = (ko_basis*)calloc(1, sizeof *b);
    b->blocks = (ko_block*)calloc((size_t)(2 * nshell + 1), sizeof(ko_block));
    int offset = 0;
    long prim = 0;
    for (int s = 0; s < nshell; ++s) {
        const int t = shell_types[s];
        const int np = nprim[s];
        if (np <= 0 || np > 64) {
            set_err(err, errlen, "invalid primitive count");
            ko_basis_destroy(b);
            return NULL;
        }
        if (t == -1) {
            if (!p_coefs) {
                set_err(err, errlen, "missing P(S=P) coefficients for sp shell");
                ko_basis_destroy(b);
                return NULL;
            }
            add_block(b, shell_xyz + 3 * s, 0, np, exps + prim, coefs + prim, 0, &offset);
            add_block(b, shell_xyz + 3 * s, 1, np, exps + prim, p_coefs + prim, 0, &offset);
        } else {
            const int l = t < 0 ? -t : t;
            add_block(b, shell_xyz + 3 * s, l, np, exps + prim, coefs + prim, t <= -2, &offset);
        }
        prim += np;
    }
    b->nao = offset;
    if (declared_nbasis > 0 && offset != declared_nbasis) {
        set_err(err, errlen, "basis size reconstructed from shells does not match fchk");
        ko_basis_destroy(b);
        return NULL;
    }
    return b;
}

void ko_basis_destroy(ko_basis* b) {
    if (!b) return;
    for (int i = 0; i < b->nblocks; ++i) {
        free(b->blocks[i].exps);
        free(b->blocks[i].weights);
        free(b->blocks[i].powers);
        free(b->blocks[i].transform);
    }
    free(b->blocks);
    free(b);
}

int ko_basis_nao(const ko_basis* b) { return b->nao; }
int ko_basis_nblocks(const ko_basis* b) { return b->nblocks; }

void ko_basis_block(const ko_basis* b, int i, int* l, int* nprim, int* offset, int* count, int* pure,
                    double* cutoff_r2) {
    const ko_block* k = &b->blocks[i];
    *l = k->l;
    *nprim = k->nprim;
    *offset = k->offset;
    *count = k->count;
    *pure = k->pure;
    *cutoff_r2 = k->cutoff_r2;
}

/* ------------------------------------------------------------------ */
/* AO kernels                                                          */
/* ------------------------------------------------------------------ */

static inline double sq_norm3(double x, double y, double z) { return x * x + y * y + z * z; }

/* src/basis_evaluator.cpp:413-488 (one point) */
static void ao_values_point(const ko_basis* b, const double* pt, double* out, double* radial,
                            double* cart) {
    for (int s = 0; s < b->nblocks; ++s) {
        const ko_block* blk = &b->blocks[s];
        const double rx = pt[0] - blk->origin[0], ry = pt[1] - blk->origin[1],
                     rz = pt[2] - blk->origin[2];
        const double r2 = sq_norm3(rx, ry, rz);
        if (r2 > blk->cutoff_r2) {
            for (int k = 0; k < blk->count; ++k) out[blk->offset + k] = 0.0;
            continue;
        }
        for (int p = 0; p < blk->nprim; ++p) radial[p] = exp(-blk->exps[p] * r2);
        double xp[32], yp[32], zp[32];
        xp[0] = yp[0] = zp[0] = 1.0;
        for (int n = 1; n <= blk->l; ++n) {
            xp[n] = xp[n - 1] * rx;
            yp[n] = yp[n - 1] * ry;
            zp[n] = zp[n - 1] * rz;
        }
        for (int k = 0; k < blk->ncart; ++k) {
            const int* pw = blk->powers[k];
            const double polynomial = (xp[pw[0]] * yp[pw[1]]) * zp[pw[2]];
            double radial_sum = 0.0;
            for (int p = 0; p < blk->nprim; ++p) radial_sum += blk->weights[k * blk->nprim + p] * radial[p];
            cart[k] = polynomial * radial_sum;
        }
        if (!blk->pure) {
            for (int k = 0; k < blk->ncart; ++k) out[blk->offset + k] = cart[k];
        } else {
            for (int m = 0; m < blk->count; ++m) {
                double s2 = 0.0;
                for (int k = 0; k < blk->ncart; ++k) s2 += blk->transform[m * blk->ncart + k] * cart[k];
                out[blk->offset + m] = s2;
            }
        }
    }
}

void ko_ao_values_batch(const ko_basis* b, const double* pts, int npts, double* out) {
    double radial[64], cart[128];
    for (int j = 0; j < npts; ++j) ao_values_point(b, pts + 3 * j, out + (long)j * b->nao, radial, cart);
}

/* src/basis_evaluator.cpp:512-643 */
void ko_ao_derivatives_batch(const ko_basis* b, const double* pts, int npts, int order, double* out) {
    const int panels = order == 2 ? 10 : 4;
    const long n = b->nao;
    const int degrees = b->max_l + 1;
    double radial[64];
    double* factors = (double*)malloc(sizeof(double) * (size_t)(b->max_prim * 3 * degrees * 3));
    double powers[3][32];
    double* scratch = (double*)malloc(sizeof(double) * (size_t)b->max_cart * 10);
#define FACTOR(p, axis, m) (&factors[(((p) * 3 + (axis)) * degrees + (m)) * 3])
    for (int s = 0; s < b->nblocks; ++s) {
        const ko_block* blk = &b->blocks[s];
        const int l_shell = blk->l;
        for (int j = 0; j < npts; ++j) {
            const double* pt = pts + 3 * j;
            const double r[3] = {pt[0] - blk->origin[0], pt[1] - blk->origin[1], pt[2] - blk->origin[2]};
            const double r2 = sq_norm3(r[0], r[1], r[2]);
            if (!(r2 <= blk->cutoff_r2)) {
                for (int c = 0; c < panels; ++c)
                    for (int k = 0; k < blk->count; ++k) out[((long)c * npts + j) * n + blk->offset + k] = 0.0;
                continue;
            }
            for (int p = 0; p < blk->nprim; ++p) radial[p] = exp(-blk->exps[p] * r2);
            for (int axis = 0; axis < 3; ++axis) {
                powers[axis][0] = 1.0;
                for (int m = 1; m <= l_shell; ++m) powers[axis][m] = powers[axis][m - 1] * r[axis];
            }
            for (int p = 0; p < blk->nprim; ++p) {
                const double a = blk->exps[p];
                for (int axis = 0; axis < 3; ++axis) {
                    const double* xp = powers[axis];
                    const double x = r[axis];
                    for (int l = 0; l <= l_shell; ++l) {
                        double* f = FACTOR(p, axis, l);
                        const double xl = xp[l];
                        f[0] = xl;
                        f[1] = (l ? l * xp[l - 1] : 0.0) - 2.0 * a * x * xl;
                        f[2] = order == 2 ? (l >= 2 ? l * (l - 1) * xp[l - 2] : 0.0) -
                                                2.0 * a * (2 * l + 1) * xl + 4.0 * a * a * x * x * xl
                                          : 0.0;
                    }
                }
            }
            for (int k = 0; k < blk->ncart; ++k) {
                const int* pw = blk->powers[k];
                double sums[10] = {0};
                for (int p = 0; p < blk->nprim; ++p) {
                    const double weight = blk->weights[k * blk->nprim + p] * radial[p];
                    const double* fx = FACTOR(p, 0, pw[0]);
                    const double* fy = FACTOR(p, 1, pw[1]);
                    const double* fz = FACTOR(p, 2, pw[2]);
                    sums[0] += weight * fx[0] * fy[0] * fz[0];
                    sums[1] += weight * fx[1] * fy[0] * fz[0];
                    sums[2] += weight * fx[0] * fy[1] * fz[0];
                    sums[3] += weight * fx[0] * fy[0] * fz[1];
                    if (order == 2) {
                        sums[4] += weight * fx[2] * fy[0] * fz[0];
                        sums[5] += weight * fx[1] * fy[1] * fz[0];
                        sums[6] += weight * fx[1] * fy[0] * fz[1];
                        sums[7] += weight * fx[0] * fy[2] * fz[0];
                        sums[8] += weight * fx[0] * fy[1] * fz[1];
                        sums[9] += weight * fx[0] * fy[0] * fz[2];
                    }
                }
                for (int c = 0; c < panels; ++c) scratch[k * 10 + c] = sums[c];
            }
            for (int c = 0; c < panels; ++c) {
                double* col = out + ((long)c * npts + j) * n + blk->offset;
                if (!blk->pure) {
                    for (int k = 0; k < blk->ncart; ++k) col[k] = scratch[k * 10 + c];
                } else {
                    for (int m = 0; m < blk->count; ++m) {
                        double s2 = 0.0;
                        for (int k = 0; k < blk->ncart; ++k)
                            s2 += blk->transform[m * blk->ncart + k] * scratch[k * 10 + c];
                        col[m] = s2;
                    }
                }
            }
        }
    }
#undef FACTOR
    free(factors);
    free(scratch);
}

void ko_significant_aos(const double* ao, int rows, long cols, double threshold, unsigned char* keep) {
    if (threshold == 0.0 || cols == 0) {
        for (int r = 0; r < rows; ++r) keep[r] = 1;
        return;
    }
    for (int r = 0; r < rows; ++r) {
        double largest = fabs(ao[r]);
        for (long c = 1; c < cols; ++c) {
            const double v = fabs(ao[c * rows + r]);
            if (v > largest) largest = v;
        }
        keep[r] = largest > threshold;
    }
}

/* ------------------------------------------------------------------ */
/* Density kernels                                                     */
/* ------------------------------------------------------------------ */

static const int hessian_column[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

static void dd_zero(ko_dd* d) { memset(d, 0, sizeof *d); }

static double trace3(const double* h) { return h[0] + h[4] + h[8]; }

/* combine, src/density.cpp:50-60 */
static ko_dd combine(const ko_dd* a, const ko_dd* b, double sign, double scale) {
    ko_dd d;
    d.value = scale * (a->value + sign * b->value);
    for (int i = 0; i < 3; ++i) d.grad[i] = scale * (a->grad[i] + sign * b->grad[i]);
    for (int i = 0; i < 9; ++i) d.hess[i] = scale * (a->hess[i] + sign * b->hess[i]);
    d.lap = trace3(d.hess);
    d.tau = scale * (a->tau + sign * b->tau);
    for (int i = 0; i < 3; ++i) d.tau_axes[i] = scale * (a->tau_axes[i] + sign * b->tau_axes[i]);
    return d;
}

static int block_count(long count, long block) { return (int)(count / block + (count % block != 0)); }

/* Rows `kept` (m of them) of the panels (nao x (panels*b), column-major) as
 * [panel][row][point] with points contiguous. */
static void gather_panels(const double* all, int nao, int panels, int b, const int* kept, int m,
                          double* dst) {
    for (int c = 0; c < panels; ++c)
        for (int r = 0; r < m; ++r)
            for (int j = 0; j < b; ++j)
                dst[((long)c * m + r) * b + j] = all[((long)c * b + j) * nao + kept[r]];
}

/* out[i][j] = sum_r coef[kept r][i] * panel[r][j]: one AO-MO projection.
 * coef is n x o column-major (MO i is column i). */
static void project_panel(const double* coef, int n, int o, const int* kept, int m,
                          const double* panel, int b, double* out) {
    memset(out, 0, sizeof(double) * (size_t)o * (size_t)b);
    for (int r = 0; r < m; ++r) {
        const double* prow = panel + (long)r * b;
        for (int i = 0; i < o; ++i) {
            const double c = coef[(long)i * n + kept[r]];
            double* orow = out + (long)i * b;
            for (int j = 0; j < b; ++j) orow[j] += c * prow[j];
        }
    }
}

/* contract (AO-MO), src/density.cpp:289-308; v[a] is o x b row-major */
static ko_dd contract_mo(double* const* v, int o, int b, int j, int ao_order) {
    ko_dd d;
    dd_zero(&d);
    if (o == 0) return d;
    double s = 0.0;
    for (int i = 0; i < o; ++i) s += v[0][(long)i * b + j] * v[0][(long)i * b + j];
    d.value = s;
    if (ao_order == 0) return d;
    for (int a = 0; a < 3; ++a) {
        double g = 0.0, t = 0.0;
        for (int i = 0; i < o; ++i) {
            g += v[0][(long)i * b + j] * v[a + 1][(long)i * b + j];
            t += v[a + 1][(long)i * b + j] * v[a + 1][(long)i * b + j];
        }
        d.grad[a] = 2.0 * g;
        d.tau_axes[a] = 0.5 * t;
        d.tau += d.tau_axes[a];
        if (ao_order == 2)
            for (int c = a; c < 3; ++c) {
                const double* vh = v[4 + hessian_column[a][c]];
                double h1 = 0.0, h2 = 0.0;
                for (int i = 0; i < o; ++i) {
                    h1 += v[0][(long)i * b + j] * vh[(long)i * b + j];
                    h2 += v[a + 1][(long)i * b + j] * v[c + 1][(long)i * b + j];
                }
                const double value = 2.0 * (h1 + h2);
                d.hess[a * 3 + c] = d.hess[c * 3 + a] = value;
            }
    }
    d.lap = trace3(d.hess);
    return d;
}

int ko_density_derivatives_mo(const ko_molecule* m, const double* pts, long npts, long block,
                              int ao_order, double threshold, ko_dd* const out[4]) {
    if (!m->ao_mo_eligible) return -1;
    if (ao_order < 0 || ao_order > 2 || block <= 0 || block > 65536) return -2;
    const int need_a = out[1] || out[0] || out[3];
    const int need_b = out[2] || out[0] || out[3];
    if (npts == 0 || !(out[0] || out[1] || out[2] || out[3])) return 0;
    const ko_basis* bs = m->basis;
    const int n = bs->nao;
    const int unrestricted = m->c_beta != NULL;
    const double* cb = unrestricted ? m->c_beta : m->c_alpha;
    const int beta_is_alpha = need_a && need_b && !unrestricted && m->nalpha == m->nbeta;
    const int panels = ao_order == 0 ? 1 : (ao_order == 1 ? 4 : 10);
    const int nblk = block_count(npts, block);
    const long cap = block < npts ? block : npts;
#pragma omp parallel
    {
        double* all = (double*)malloc(sizeof(double) * (size_t)n * panels * cap);
        double* kept_panels = (double*)malloc(sizeof(double) * (size_t)n * panels * cap);
        int* kept = (int*)malloc(sizeof(int) * (size_t)n);
        unsigned char* keep = (unsigned char*)malloc((size_t)n);
        const int omax = (m->nalpha > m->nbeta ? m->nalpha : m->nbeta);
        double* va[10];
        double* vb[10];
        for (int a = 0; a < 10; ++a) {
            va[a] = (double*)malloc(sizeof(double) * (size_t)(omax > 0 ? omax : 1) * cap);
            vb[a] = (double*)malloc(sizeof(double) * (size_t)(omax > 0 ? omax : 1) * cap);
        }
#pragma omp for schedule(dynamic)
        for (int blk = 0; blk < nblk; ++blk) {
            const long start = (long)blk * block;
            const int b = (int)((npts - start) < block ? (npts - start) : block);
            if (ao_order == 0)
                ko_ao_values_batch(bs, pts + 3 * start, b, all);
            else
                ko_ao_derivatives_batch(bs, pts + 3 * start, b, ao_order, all);
            ko_significant_aos(all, n, (long)panels * b, threshold, keep);
            int mk = 0;
            for (int r = 0; r < n; ++r)
                if (keep[r]) kept[mk++] = r;
            gather_panels(all, n, panels, b, kept, mk, kept_panels);
            if (need_a && m->nalpha > 0)
                for (int a = 0; a < panels; ++a)
                    project_panel(m->c_alpha, n, m->nalpha, kept, mk, kept_panels + (long)a * mk * b, b, va[a]);
            if (need_b && !beta_is_alpha && m->nbeta > 0)
                for (int a = 0; a < panels; ++a)
                    project_panel(cb, n, m->nbeta, kept, mk, kept_panels + (long)a * mk * b, b, vb[a]);
            for (int j = 0; j < b; ++j) {
                ko_dd alpha, beta;
                dd_zero(&alpha);
                dd_zero(&beta);
                if (need_a) alpha = contract_mo(va, m->nalpha, b, j, ao_order);
                if (beta_is_alpha)
                    beta = alpha;
                else if (need_b)
                    beta = contract_mo(vb, m->nbeta, b, j, ao_order);
                const long slot = start + j;
                if (out[1]) out[1][slot] = alpha;
                if (out[2]) out[2][slot] = beta;
                if (out[0]) out[0][slot] = combine(&alpha, &beta, 1.0, 1.0);
                if (out[3]) out[3][slot] = combine(&alpha, &beta, -1.0, 1.0);
            }
        }
        for (int a = 0; a < 10; ++a) {
            free(va[a]);
            free(vb[a]);
        }
        free(all);
        free(kept_panels);
        free(kept);
        free(keep);
    }
    return 0;
}

/* y = Pk * panels[0..4) with Pk = P(kept, kept): y[c][r][j] */
static void p_product(const double* P, int n, const int* kept, int mk, const double* kp, int b,
                      int cols_panels, double* y, double* prow_buf) {
    for (int r = 0; r < mk; ++r) {
        for (int s = 0; s < mk; ++s) prow_buf[s] = P[(long)kept[s] * n + kept[r]];
        for (int c = 0; c < cols_panels; ++c) {
            double* yr = y + ((long)c * mk + r) * b;
            for (int j = 0; j < b; ++j) yr[j] = 0.0;
            for (int s = 0; s < mk; ++s) {
                const double pv = prow_buf[s];
                const double* ph = kp + ((long)c * mk + s) * b;
                for (int j = 0; j < b; ++j) yr[j] += pv * ph[j];
            }
        }
    }
}

/* contract_derivatives, src/density.cpp:26-44; kp[c][r][j], y[c][r][j] */
static ko_dd contract_p(const double* kp, const double* y, int mk, int b, int j, int ao_order) {
    ko_dd d;
    dd_zero(&d);
#define KP(c, r) kp[((long)(c) * mk + (r)) * b + j]
#define YP(c, r) y[((long)(c) * mk + (r)) * b + j]
    double s = 0.0;
    for (int r = 0; r < mk; ++r) s += KP(0, r) * YP(0, r);
    d.value = s;
    for (int a = 0; a < 3; ++a) {
        double g = 0.0, t = 0.0;
        for (int r = 0; r < mk; ++r) {
            g += KP(a + 1, r) * YP(0, r);
            t += KP(a + 1, r) * YP(a + 1, r);
        }
        d.grad[a] = 2.0 * g;
        d.tau_axes[a] = 0.5 * t;
        d.tau += d.tau_axes[a];
        if (ao_order == 2)
            for (int c = a; c < 3; ++c) {
                double h1 = 0.0, h2 = 0.0;
                for (int r = 0; r < mk; ++r) {
                    h1 += KP(4 + hessian_column[a][c], r) * YP(0, r);
                    h2 += KP(a + 1, r) * YP(c + 1, r);
                }
                const double v = 2.0 * (h1 + h2);
                d.hess[a * 3 + c] = d.hess[c * 3 + a] = v;
            }
    }
#undef KP
#undef YP
    d.lap = trace3(d.hess);
    return d;
}

int ko_density_derivatives_shared(const ko_molecule* m, const double* pts, long npts, long block,
                                  int ao_order, double threshold, ko_dd* const out[4]) {
    if (ao_order != 1 && ao_order != 2) return -2;
    if (block <= 0) return -2;
    const int total_needed = out[0] || out[1] || out[2];
    const int spin_needed = out[3] || out[1] || out[2];
    if (npts == 0 || !(total_needed || spin_needed)) return 0;
    const ko_basis* bs = m->basis;
    const int n = bs->nao;
    const int panels = ao_order == 2 ? 10 : 4;
    const int nblk = block_count(npts, block);
    const long cap = block < npts ? block : npts;
#pragma omp parallel
    {
        double* all = (double*)malloc(sizeof(double) * (size_t)n * panels * cap);
        double* kp = (double*)malloc(sizeof(double) * (size_t)n * panels * cap);
        double* yt = (double*)malloc(sizeof(double) * (size_t)n * 4 * cap);
        double* ys = (double*)malloc(sizeof(double) * (size_t)n * 4 * cap);
        double* prow = (double*)malloc(sizeof(double) * (size_t)n);
        int* kept = (int*)malloc(sizeof(int) * (size_t)n);
        unsigned char* keep = (unsigned char*)malloc((size_t)n);
#pragma omp for schedule(dynamic)
        for (int blk = 0; blk < nblk; ++blk) {
            const long start = (long)blk * block;
            const int b = (int)((npts - start) < block ? (npts - start) : block);
            ko_ao_derivatives_batch(bs, pts + 3 * start, b, ao_order, all);
            ko_significant_aos(all, n, (long)panels * b, threshold, keep);
            int mk = 0;
            for (int r = 0; r < n; ++r)
                if (keep[r]) kept[mk++] = r;
            gather_panels(all, n, panels, b, kept, mk, kp);
            if (total_needed) p_product(m->p_total, n, kept, mk, kp, b, 4, yt, prow);
            if (spin_needed) p_product(m->p_spin, n, kept, mk, kp, b, 4, ys, prow);
            for (int j = 0; j < b; ++j) {
                ko_dd t, s;
                dd_zero(&t);
                dd_zero(&s);
                if (total_needed) t = contract_p(kp, yt, mk, b, j, ao_order);
                if (spin_needed) s = contract_p(kp, ys, mk, b, j, ao_order);
                const long slot = start + j;
                if (out[0]) out[0][slot] = t;
                if (out[3]) out[3][slot] = s;
                if (out[1]) out[1][slot] = combine(&t, &s, 1.0, 0.5);
                if (out[2]) out[2][slot] = combine(&t, &s, -1.0, 0.5);
            }
        }
        free(all);
        free(kp);
        free(yt);
        free(ys);
        free(prow);
        free(kept);
        free(keep);
    }
    return 0;
}

int ko_densities_blocked(const ko_molecule* m, const double* pts, long npts, long block,
                         double threshold, int component, double* out) {
    const ko_basis* bs = m->basis;
    const int n = bs->nao;
    if (block <= 0 || block > 65536) return -2;
    /* select_density_matrix, src/density_matrix.hpp:12-24 */
    double* pm = NULL;
    const double* P = NULL;
    if (component == 0)
        P = m->p_total;
    else if (component == 3)
        P = m->p_spin;
    else {
        pm = (double*)malloc(sizeof(double) * (size_t)n * n);
        for (long i = 0; i < (long)n * n; ++i)
            pm[i] = component == 1 ? 0.5 * (m->p_total[i] + m->p_spin[i]) : 0.5 * (m->p_total[i] - m->p_spin[i]);
        P = pm;
    }
    const int nblk = block_count(npts, block);
    const long cap = block < npts ? block : npts;
#pragma omp parallel
    {
        double* phi = (double*)malloc(sizeof(double) * (size_t)n * cap);
        double* kp = (double*)malloc(sizeof(double) * (size_t)n * cap);
        double* y = (double*)malloc(sizeof(double) * (size_t)n * cap);
        double* prow = (double*)malloc(sizeof(double) * (size_t)n);
        int* kept = (int*)malloc(sizeof(int) * (size_t)n);
        unsigned char* keep = (unsigned char*)malloc((size_t)n);
#pragma omp for schedule(dynamic)
        for (int blk = 0; blk < nblk; ++blk) {
            const long start = (long)blk * block;
            const int b = (int)((npts - start) < block ? (npts - start) : block);
            ko_ao_values_batch(bs, pts + 3 * start, b, phi);
            ko_significant_aos(phi, n, b, threshold, keep);
            int mk = 0;
            for (int r = 0; r < n; ++r)
                if (keep[r]) kept[mk++] = r;
            gather_panels(phi, n, 1, b, kept, mk, kp);
            p_product(P, n, kept, mk, kp, b, 1, y, prow);
            for (int j = 0; j < b; ++j) {
                double s = 0.0;
                for (int r = 0; r < mk; ++r) s += kp[(long)r * b + j] * y[(long)r * b + j];
                out[start + j] = s;
            }
        }
        free(phi);
        free(kp);
        free(y);
        free(prow);
        free(kept);
        free(keep);
    }
    free(pm);
    return 0;
}

int ko_orbitals(const ko_molecule* m, const double* pts, long npts, int channel, const long* indices,
                int nidx, double* const* out) {
    const ko_basis* bs = m->basis;
    const int n = bs->nao;
    const double* coef = (channel == 1 && m->c_beta) ? m->c_beta : m->c_alpha;
    const int nmo = (channel == 1 && m->c_beta) ? m->nmo_beta : m->nmo_alpha;
    for (int i = 0; i < nidx; ++i)
        if (indices[i] < 1 || indices[i] > nmo) return -3;
    const long block = 128;
    const int nblk = block_count(npts, block);
#pragma omp parallel
    {
        double* phi = (double*)malloc(sizeof(double) * (size_t)n * block);
#pragma omp for schedule(dynamic)
        for (int blk = 0; blk < nblk; ++blk) {
            const long start = (long)blk * block;
            const int b = (int)((npts - start) < block ? (npts - start) : block);
            ko_ao_values_batch(bs, pts + 3 * start, b, phi);
            for (int q = 0; q < nidx; ++q) {
                const double* c = coef + (long)(indices[q] - 1) * n;
                for (int j = 0; j < b; ++j) {
                    double s = 0.0;
                    for (int r = 0; r < n; ++r) s += c[r] * phi[(long)j * n + r];
                    out[q][start + j] = s;
                }
            }
        }
        free(phi);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Derived fields, src/evaluator.cpp:117-353                            */
/* ------------------------------------------------------------------ */

static double fermi_constant(void) { return 0.3 * pow(6.0 * KO_PI * KO_PI, 2.0 / 3.0); }

static double elf_channels(const ko_dd* const* ch, int nch) {
    const double fermi = fermi_constant();
    double pauli = 0.0, uniform = 0.0;
    for (int i = 0; i < nch; ++i) {
        const ko_dd* d = ch[i];
        if (!(d->value > 0.0)) continue;
        const double g2 = d->grad[0] * d->grad[0] + d->grad[1] * d->grad[1] + d->grad[2] * d->grad[2];
        pauli += d->tau - g2 / (8.0 * d->value);
        uniform += fermi * pow(d->value, 5.0 / 3.0);
    }
    if (!(uniform > 0.0)) return 0.0;
    const double chi = pauli / uniform;
    return 1.0 / (1.0 + chi * chi);
}

static double lol_channels(const ko_dd* const* ch, int nch) {
    const double fermi = fermi_constant();
    double tau = 0.0, uniform = 0.0;
    for (int i = 0; i < nch; ++i) {
        tau += ch[i]->tau;
        if (ch[i]->value > 0.0) uniform += fermi * pow(ch[i]->value, 5.0 / 3.0);
    }
    if (!(uniform > 0.0)) return 0.0;
    if (!(tau > 0.0)) return 1.0;
    return uniform / (tau + uniform);
}

static double gradient_expansion(const ko_dd* const* ch, int nch, int lol) {
    const double fermi = fermi_constant();
    double uniform = 0.0, pauli = 0.0, kinetic = 0.0;
    for (int i = 0; i < nch; ++i) {
        const ko_dd* d = ch[i];
        if (!(d->value > 0.0)) continue;
        const double reference = fermi * pow(d->value, 5.0 / 3.0);
        const double g2 = d->grad[0] * d->grad[0] + d->grad[1] * d->grad[1] + d->grad[2] * d->grad[2];
        const double weizsacker = g2 / d->value;
        uniform += reference;
        pauli += reference - weizsacker / 9.0 + d->lap / 6.0;
        kinetic += reference + weizsacker / 72.0 + d->lap / 6.0;
    }
    if (!(uniform > 0.0)) return 0.0;
    if (lol) {
        const double den = kinetic + uniform;
        return den != 0.0 ? uniform / den : 0.0;
    }
    const double chi = pauli / uniform;
    return 1.0 / (1.0 + chi * chi);
}

static double grad_norm(const ko_dd* d) {
    return sqrt(d->grad[0] * d->grad[0] + d->grad[1] * d->grad[1] + d->grad[2] * d->grad[2]);
}

static double reduced_gradient(const ko_dd* d) {
    const double scale = 2.0 * cbrt(3.0 * KO_PI * KO_PI);
    if (!(d->value > 0.0)) return 100.0;
    const double den = scale * pow(d->value, 4.0 / 3.0);
    const double norm = grad_norm(d);
    if (!(den > 0.0) || !(norm < 100.0 * den)) return 100.0;
    return norm / den;
}

/* Eigenvalues of a symmetric 3x3 matrix by cyclic Jacobi rotations, sorted
 * ascending (stands in for Eigen's SelfAdjointEigenSolver). */
static void sym3_eigenvalues(const double* h, double* ev) {
    double a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = h[i * 3 + j];
    for (int sweep = 0; sweep < 64; ++sweep) {
        const double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        if (off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                if (a[p][q] == 0.0) continue;
                const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    const double akp = a[k][p], akq = a[k][q];
                    a[k][p] = c * akp - s * akq;
                    a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    const double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = c * apk - s * aqk;
                    a[q][k] = s * apk + c * aqk;
                }
            }
    }
    ev[0] = a[0][0];
    ev[1] = a[1][1];
    ev[2] = a[2][2];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2 - i; ++j)
            if (ev[j] > ev[j + 1]) {
                const double t = ev[j];
                ev[j] = ev[j + 1];
                ev[j + 1] = t;
            }
}

static double sign_lambda2(const ko_dd* d) {
    double ev[3];
    sym3_eigenvalues(d->hess, ev);
    return ev[1] < 0.0 ? -d->value : d->value;
}

static double iri(const ko_dd* d) {
    if (!(d->value > 0.0)) return 100.0;
    const double v = grad_norm(d) / pow(d->value, 1.1);
    return v < 100.0 ? v : 100.0;
}

static double dori(const ko_dd* d) {
    if (!(d->value > 0.0)) return 0.0;
    double q[3];
    for (int a = 0; a < 3; ++a) q[a] = d->grad[a] / d->value;
    const double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    if (!(q2 > 0.0)) return 1.0;
    double w[3];
    for (int a = 0; a < 3; ++a) {
        const double hq = d->hess[a * 3 + 0] * q[0] + d->hess[a * 3 + 1] * q[1] + d->hess[a * 3 + 2] * q[2];
        w[a] = hq / d->value - q2 * q[a];
    }
    const double theta = 4.0 * (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) / (q2 * q2 * q2);
    if (!isfinite(theta)) return 1.0;
    return theta / (1.0 + theta);
}

static int channels_of(int kind) {
    switch (kind) {
    case 1: case 24: case 30: case 31: return 3;
    case 2: case 25: return 6;
    default: return 1;
    }
}

/* store_block, src/evaluator.cpp:248-353: one property at one point */
static void store_point(const ko_property* key, ko_dd* const* comp, long p, long npts, double* out) {
    const int kind = key->kind;
    if ((kind == 6 || kind == 10 || kind == 35 || kind == 36) && key->component == 0) {
        const ko_dd* ch[2] = {&comp[1][p], &comp[2][p]};
        double v;
        if (kind == 6) v = elf_channels(ch, 2);
        else if (kind == 10) v = lol_channels(ch, 2);
        else v = gradient_expansion(ch, 2, kind == 36);
        out[p] = v;
        return;
    }
    if (kind == 16) {
        const double t = comp[0][p].value;
        out[p] = t > 0.0 ? comp[3][p].value / t : 0.0;
        return;
    }
    const ko_dd* d = &comp[key->component][p];
    const ko_dd* one[1] = {d};
    switch (kind) {
    case 0: out[p] = d->value; break;
    case 1: for (int a = 0; a < 3; ++a) out[a * npts + p] = d->grad[a]; break;
    case 2:
        out[0 * npts + p] = d->hess[0];
        out[1 * npts + p] = d->hess[1];
        out[2 * npts + p] = d->hess[2];
        out[3 * npts + p] = d->hess[4];
        out[4 * npts + p] = d->hess[5];
        out[5 * npts + p] = d->hess[8];
        break;
    case 3: out[p] = d->lap; break;
    case 4: out[p] = d->tau; break;
    case 6: out[p] = elf_channels(one, 1); break;
    case 7: out[p] = reduced_gradient(d); break;
    case 8: out[p] = sign_lambda2(d); break;
    case 10: out[p] = lol_channels(one, 1); break;
    case 35: out[p] = gradient_expansion(one, 1, 0); break;
    case 36: out[p] = gradient_expansion(one, 1, 1); break;
    case 11: out[p] = iri(d); break;
    case 12: out[p] = dori(d); break;
    case 13: out[p] = d->tau - 0.25 * d->lap; break;
    case 14: out[p] = 0.25 * d->lap - 2.0 * d->tau; break;
    case 15: out[p] = 0.25 * d->lap - d->tau; break;
    case 30: for (int a = 0; a < 3; ++a) out[a * npts + p] = d->tau_axes[a]; break;
    case 31: for (int a = 0; a < 3; ++a) out[a * npts + p] = d->tau_axes[a] - 0.25 * d->hess[a * 4]; break;
    case 32: out[p] = d->tau > 0.0 ? fabs(0.25 * d->lap - 2.0 * d->tau) / d->tau : 0.0; break;
    case 33: out[p] = d->value > 0.0 ? (0.25 * d->lap - d->tau) / d->value : 0.0; break;
    case 34: out[p] = d->value > 0.0 ? d->tau / d->value : 0.0; break;
    case 17: out[p] = d->value > 0.0 ? -d->value * log(d->value) : 0.0; break;
    case 18: {
        const double g2 = d->grad[0] * d->grad[0] + d->grad[1] * d->grad[1] + d->grad[2] * d->grad[2];
        out[p] = d->value > 0.0 ? g2 / d->value : 0.0;
        break;
    }
    default: break;
    }
}

/* ------------------------------------------------------------------ */
/* Evaluation plan and backend choice                                  */
/* ------------------------------------------------------------------ */

typedef struct {
    int density, gradient, hessian, laplacian, tau, elf_input, reduced_gradient, sign_lambda2,
        lol_input, gradient_expansion_input, gradient_input, hessian_input, energy_input, tau_input,
        value_input, esp;
} ko_cplan;

static int cplan_derivatives(const ko_cplan* c) {
    return c->gradient || c->hessian || c->laplacian || c->tau || c->elf_input || c->reduced_gradient ||
           c->sign_lambda2 || c->lol_input || c->gradient_input || c->hessian_input || c->energy_input ||
           c->tau_input || c->gradient_expansion_input || c->value_input;
}

static int cplan_order(const ko_cplan* c) {
    if (c->hessian || c->laplacian || c->sign_lambda2 || c->hessian_input || c->energy_input ||
        c->gradient_expansion_input)
        return 2;
    if (c->gradient || c->tau || c->elf_input || c->reduced_gradient || c->lol_input || c->gradient_input ||
        c->tau_input || c->value_input)
        return 1;
    return c->density ? 0 : -1;
}

/* EvaluationPlan::from, src/evaluation_plan.hpp:153-273 */
static int make_plan(const ko_property* props, int nprops, ko_cplan comp[4], int* orbitals, int* max_order,
                     char* err, int errlen) {
    memset(comp, 0, sizeof(ko_cplan) * 4);
    *orbitals = 0;
    *max_order = -1;
    for (int i = 0; i < nprops; ++i) {
        const ko_property* p = &props[i];
        if (p->kind == 5 || p->kind == 24 || p->kind == 25) {
            if (p->orbital_index == 0) {
                set_err(err, errlen, "orbital indices are one-based");
                return -1;
            }
            *orbitals = 1;
            if (*max_order < 0) *max_order = 0;
            continue;
        }
        if (p->component < 0 || p->component > 3) {
            set_err(err, errlen, "invalid density spin component");
            return -1;
        }
        ko_cplan* c = &comp[p->component];
        const int total = p->component == 0;
        switch (p->kind) {
        case 0: c->density = 1; break;
        case 1: c->gradient = 1; break;
        case 2: c->hessian = 1; break;
        case 3: c->laplacian = 1; break;
        case 4: c->tau = 1; break;
        case 6: case 10: case 35: case 36:
            if (p->component == 3) {
                set_err(err, errlen, "not defined for the spin-difference density");
                return -1;
            }
            if (total) {
                if (p->kind == 6) comp[1].elf_input = comp[2].elf_input = 1;
                else if (p->kind == 10) comp[1].lol_input = comp[2].lol_input = 1;
                else comp[1].gradient_expansion_input = comp[2].gradient_expansion_input = 1;
            } else {
                if (p->kind == 6) c->elf_input = 1;
                else if (p->kind == 10) c->lol_input = 1;
                else c->gradient_expansion_input = 1;
            }
            break;
        case 7: case 8: case 9: case 11: case 12: case 14: case 15: case 32: case 33: case 34: case 17:
        case 18:
            if (!total) {
                set_err(err, errlen, "is defined only for the total density");
                return -1;
            }
            if (p->kind == 7) c->reduced_gradient = 1;
            else if (p->kind == 8) c->sign_lambda2 = 1;
            else if (p->kind == 9) c->esp = 1;
            else if (p->kind == 11 || p->kind == 17 || p->kind == 18) c->gradient_input = 1;
            else if (p->kind == 12) c->hessian_input = 1;
            else if (p->kind == 34) c->tau_input = 1;
            else c->energy_input = 1;
            break;
        case 13: case 31: c->energy_input = 1; break;
        case 30: c->tau_input = 1; break;
        case 16:
            if (p->component != 3) {
                set_err(err, errlen, "the spin polarization is defined only for the spin component");
                return -1;
            }
            comp[0].value_input = 1;
            c->value_input = 1;
            break;
        default:
            set_err(err, errlen, "unsupported property kind");
            return -1;
        }
    }
    for (int c = 0; c < 4; ++c) {
        const int o = cplan_order(&comp[c]);
        if (o > *max_order) *max_order = o;
    }
    return 0;
}

/* choose_backend, src/automatic_backend.hpp:38-50: 1 AO_P, 2 AO_MO */
static int choose_backend(int requested, int eligible, const ko_cplan comp[4]) {
    if (requested == 1) return 1;
    if (requested == 2) return eligible ? 2 : -1;
    if (!eligible) return 1;
    for (int c = 0; c < 4; ++c)
        if (cplan_order(&comp[c]) >= 0) return 2;
    return 1;
}

void ko_grid_points(const double* origin, const double* steps, const int* counts, long start, long count,
                    double* out) {
    const long ny = counts[1], nz = counts[2];
    for (long q = 0; q < count; ++q) {
        const long linear = start + q;
        const double i = (double)(linear / (ny * nz)), j = (double)((linear / nz) % ny),
                     k = (double)(linear % nz);
        for (int r = 0; r < 3; ++r)
            out[3 * q + r] = origin[r] + ((steps[0 * 3 + r] * i + steps[1 * 3 + r] * j) + steps[2 * 3 + r] * k);
    }
}

int ko_evaluate(const ko_molecule* m, const ko_options* opt, const double* origin, const double* steps,
                const int* counts, const double* points, long npoints, const ko_property* props,
                int nprops, double* const* outputs, int* backend_used, char* err, int errlen) {
    ko_cplan comp[4];
    int orbitals = 0, max_order = -1;
    if (opt->block_size <= 0 || opt->block_size > 65536) {
        set_err(err, errlen, "evaluation block_size must be in [1, 65536]");
        return -1;
    }
    if (make_plan(props, nprops, comp, &orbitals, &max_order, err, errlen)) return -1;
    const int backend = choose_backend(opt->backend, m->ao_mo_eligible, comp);
    if (backend < 0) {
        set_err(err, errlen, "AO_MO requested for ineligible orbital representation");
        return -1;
    }
    if (backend_used) *backend_used = backend;
    const int grid = origin != NULL;
    long n = npoints;
    double* pts = NULL;
    if (grid) {
        n = (long)counts[0] * counts[1] * counts[2];
        pts = (double*)malloc(sizeof(double) * 3 * (size_t)n);
        ko_grid_points(origin, steps, counts, 0, n, pts);
    } else {
        pts = (double*)malloc(sizeof(double) * 3 * (size_t)n);
        memcpy(pts, points, sizeof(double) * 3 * (size_t)n);
    }
    /* Point path, src/evaluator.cpp:366-389,638-657 */
    int uses[4] = {0};
    int any = 0;
    for (int c = 0; c < 4; ++c) {
        uses[c] = cplan_derivatives(&comp[c]) || ((backend == 2 || !grid) && comp[c].density);
        any |= uses[c];
    }
    int status = 0;
    if (any) {
        ko_dd* dd[4] = {NULL, NULL, NULL, NULL};
        for (int c = 0; c < 4; ++c)
            if (uses[c]) dd[c] = (ko_dd*)calloc((size_t)n, sizeof(ko_dd));
        const int ao_order = grid ? max_order : (max_order > 1 ? max_order : 1);
        if (backend == 2)
            status = ko_density_derivatives_mo(m, pts, n, opt->block_size, ao_order < 0 ? 0 : ao_order,
                                               opt->screening_threshold, dd);
        else
            status = ko_density_derivatives_shared(m, pts, n, opt->block_size, ao_order,
                                                   opt->screening_threshold, dd);
        if (!status)
            for (int i = 0; i < nprops; ++i) {
                const ko_property* key = &props[i];
                const int on_grid_path = grid && (key->kind == 5 || (key->kind == 0 && backend == 1));
                if (on_grid_path || key->kind == 5 || key->kind == 24 || key->kind == 25 || key->kind == 9)
                    continue;
                for (long p = 0; p < n; ++p) store_point(key, dd, p, n, outputs[i]);
            }
        for (int c = 0; c < 4; ++c) free(dd[c]);
    }
    /* Electrostatic potential pass (exact) */
    for (int i = 0; i < nprops && !status; ++i) {
        if (props[i].kind != 9) continue;
        ko_esp* e = ko_esp_create(m->basis, m->p_total, m->natoms, m->atom_xyz, m->atom_charge);
        ko_esp_evaluate(e, pts, n, outputs[i]);
        ko_esp_destroy(e);
    }
    /* Grid path, src/evaluator.cpp:754-777, and orbital amplitudes */
    for (int i = 0; i < nprops && !status; ++i) {
        const ko_property* key = &props[i];
        if (grid && key->kind == 0 && backend == 1)
            status = ko_densities_blocked(m, pts, n, opt->block_size, opt->screening_threshold,
                                          key->component, outputs[i]);
        else if (key->kind == 5) {
            double* o[1] = {outputs[i]};
            status = ko_orbitals(m, pts, n, key->channel, &key->orbital_index, 1, o);
        }
    }
    free(pts);
    if (status) set_err(err, errlen, "evaluation failed");
    return status;
}

int ko_validate_orbital_backend(int n, const double* total, const double* spin, const double* alpha,
                                int nmo_a, const double* beta, int nmo_b, int nalpha, int nbeta,
                                int unrestricted, double* errors4) {
    const double* bc = unrestricted ? beta : alpha;
    const int nmob = unrestricted ? nmo_b : nmo_a;
    if (nalpha > nmo_a || nbeta > nmob || (!unrestricted && nalpha != nbeta)) return 0;
    double te = 0, se = 0, tn = 0, rtn = 0, sn = 0, rsn = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double pa = 0.0, pb = 0.0;
            for (int k = 0; k < nalpha; ++k) pa += alpha[(long)k * n + i] * alpha[(long)k * n + j];
            for (int k = 0; k < nbeta; ++k) pb += bc[(long)k * n + i] * bc[(long)k * n + j];
            const double rt = pa + pb, rs = pa - pb;
            const double t = total[(long)j * n + i], s = spin[(long)j * n + i];
            te += (t - rt) * (t - rt);
            se += (s - rs) * (s - rs);
            tn += t * t;
            rtn += rt * rt;
            sn += s * s;
            rsn += rs * rs;
        }
    te = sqrt(te);
    se = sqrt(se);
    const double total_scale = fmax(sqrt(tn), sqrt(rtn));
    const double spin_scale = fmax(fmax(sqrt(sn), sqrt(rsn)), total_scale);
    if (errors4) {
        errors4[0] = te;
        errors4[1] = total_scale > 0 ? te / total_scale : te;
        errors4[2] = se;
        errors4[3] = spin_scale > 0 ? se / spin_scale : se;
    }
    return te <= 1e-10 + 1e-8 * total_scale && se <= 1e-10 + 1e-8 * spin_scale;
}

/* ------------------------------------------------------------------ */
/* Boys function, src/boys_function.cpp                                */
/* ------------------------------------------------------------------ */

#define KO_BOYS_MAX 32
#define KO_TAYLOR 7
#define KO_TABLE_ORDERS (KO_BOYS_MAX + KO_TAYLOR)
#define KO_TABLE_POINTS 801
static double* boys_table = NULL;

static const double* boys_table_get(void) {
#pragma omp critical(ko_boys_table)
    {
        if (!boys_table) {
            double* t = (double*)malloc(sizeof(double) * KO_TABLE_POINTS * KO_TABLE_ORDERS);
            const int top = KO_TABLE_ORDERS - 1;
            for (int i = 0; i < KO_TABLE_POINTS; ++i) {
                const double T = i * 0.05;
                const double decay = exp(-T);
                double term = 1.0 / (2.0 * top + 1.0);
                double sum = term;
                for (int k = 1; k < 10000 && term > 1e-18 * sum; ++k) {
                    term *= 2.0 * T / (2.0 * top + 2.0 * k + 1.0);
                    sum += term;
                }
                double* row = t + (long)i * KO_TABLE_ORDERS;
                row[top] = decay * sum;
                for (int m = top; m > 0; --m) row[m - 1] = (2.0 * T * row[m] + decay) / (2.0 * m - 1.0);
            }
            boys_table = t;
        }
    }
    return boys_table;
}

int ko_boys(double T, int nvalues, double* values) {
    if (nvalues <= 0 || nvalues > KO_BOYS_MAX + 1) return -1;
    if (!isfinite(T) || T < 0.0) return -1;
    const int top = nvalues - 1;
    const double decay = exp(-T);
    if (T >= 40.0) {
        values[0] = 0.5 * sqrt(KO_PI / T);
        for (int m = 0; m < top; ++m) values[m + 1] = ((2.0 * m + 1.0) * values[m] - decay) / (2.0 * T);
        return 0;
    }
    const int point = (int)lround(T / 0.05);
    const double delta = T - point * 0.05;
    const double* row = boys_table_get() + (long)point * KO_TABLE_ORDERS;
    double sum = 0.0, factor = 1.0;
    for (int k = 0; k < KO_TAYLOR; ++k) {
        sum += row[top + k] * factor;
        factor *= -delta / (k + 1.0);
    }
    values[top] = sum;
    for (int m = top; m > 0; --m) values[m - 1] = (2.0 * T * values[m] + decay) / (2.0 * m - 1.0);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Electrostatic potential, src/electrostatic_potential.cpp:17-360      */
/* ------------------------------------------------------------------ */

typedef struct {
    double exponent;
    double center[3];
    int order;
    long first;
} ko_pair;

struct ko_esp {
    long npairs, cap_pairs;
    ko_pair* pairs;
    double* coef;
    long ncoef, cap_coef;
    int max_order, side;
    int* hidx;      /* offsets of (t,u,v) for order max_order, ordered by t+u+v */
    int (*triples)[3];
    int ntriples;
    int natoms;
    double* xyz;
    double* charge;
};

static int hermite_count(int s) { return (s + 1) * (s + 2) * (s + 3) / 6; }

static int hermite_triples(int L, int (*out)[3]) {
    int n = 0;
    for (int sum = 0; sum <= L; ++sum)
        for (int t = sum; t >= 0; --t)
            for (int u = sum - t; u >= 0; --u) {
                out[n][0] = t;
                out[n][1] = u;
                out[n][2] = sum - t - u;
                ++n;
            }
    return n;
}

/* HermiteTable, src/electrostatic_potential.cpp:57-93 */
static void hermite_table(int la, int lb, double p, double pa, double pb, double* tab) {
    const int width = la + lb + 1;
    const double half = 0.5 / p;
    memset(tab, 0, sizeof(double) * (size_t)((la + 1) * (lb + 1) * width));
#define HT(i, j, t) tab[((i) * (lb + 1) + (j)) * width + (t)]
#define HG(i, j, t) (((t) < 0 || (t) > (i) + (j)) ? 0.0 : HT(i, j, t))
    HT(0, 0, 0) = 1.0;
    for (int i = 0; i < la; ++i)
        for (int t = 0; t <= i + 1; ++t) {
            double v = pa * HG(i, 0, t);
            if (t > 0) v += half * HG(i, 0, t - 1);
            if (t + 1 <= i) v += (t + 1) * HG(i, 0, t + 1);
            HT(i + 1, 0, t) = v;
        }
    for (int i = 0; i <= la; ++i)
        for (int j = 0; j < lb; ++j)
            for (int t = 0; t <= i + j + 1; ++t) {
                double v = pb * HG(i, j, t);
                if (t > 0) v += half * HG(i, j, t - 1);
                if (t + 1 <= i + j) v += (t + 1) * HG(i, j, t + 1);
                HT(i, j + 1, t) = v;
            }
#undef HT
#undef HG
}

static double hget(const double* tab, int lb, int width, int i, int j, int t) {
    if (t < 0 || t > i + j) return 0.0;
    return tab[(i * (lb + 1) + j) * width + t];
}

ko_esp* ko_esp_create(const ko_basis* b, const double* P, int natoms, const double* xyz, const double* charges) {
    ko_esp* e = (ko_esp*)calloc(1, sizeof *e);
    const int n = b->nao;
    e->natoms = natoms;
    e->xyz = (double*)malloc(sizeof(double) * 3 * (size_t)natoms);
    e->charge = (double*)malloc(sizeof(double) * (size_t)natoms);
    memcpy(e->xyz, xyz, sizeof(double) * 3 * (size_t)natoms);
    memcpy(e->charge, charges, sizeof(double) * (size_t)natoms);
    for (int i = 0; i < b->nblocks; ++i)
        if (2 * b->blocks[i].l > e->max_order) e->max_order = 2 * b->blocks[i].l;
    e->side = e->max_order + 10 + 1;
    e->triples = malloc(sizeof(int[3]) * (size_t)hermite_count(e->side));
    e->ntriples = hermite_triples(e->side - 1, e->triples);
    e->hidx = (int*)malloc(sizeof(int) * (size_t)hermite_count(e->max_order));
    for (int k = 0; k < hermite_count(e->max_order); ++k)
        e->hidx[k] = (e->triples[k][0] * e->side + e->triples[k][1]) * e->side + e->triples[k][2];
    double cart[100 * 100];
    double tmp[100 * 100];
    double* ex = (double*)malloc(sizeof(double) * 4096);
    double* ey = (double*)malloc(sizeof(double) * 4096);
    double* ez = (double*)malloc(sizeof(double) * 4096);
    double* pc = (double*)malloc(sizeof(double) * (size_t)hermite_count(e->max_order));
    for (int a = 0; a < b->nblocks; ++a) {
        const ko_block* A = &b->blocks[a];
        for (int bb = a; bb < b->nblocks; ++bb) {
            const ko_block* B = &b->blocks[bb];
            /* cart = TA^T * P(A rows, B cols) * TB, ncartA x ncartB */
            const int ra = A->count, rb = B->count;
            for (int i = 0; i < ra; ++i)
                for (int j = 0; j < rb; ++j) tmp[i * rb + j] = P[(long)(B->offset + j) * n + A->offset + i];
            double left[100 * 100];
            if (A->pure) {
                for (int k = 0; k < A->ncart; ++k)
                    for (int j = 0; j < rb; ++j) {
                        double s = 0.0;
                        for (int i = 0; i < ra; ++i) s += A->transform[i * A->ncart + k] * tmp[i * rb + j];
                        left[k * rb + j] = s;
                    }
            } else {
                memcpy(left, tmp, sizeof(double) * (size_t)(ra * rb));
            }
            const int na = A->ncart, nb = B->ncart;
            if (B->pure) {
                for (int i = 0; i < na; ++i)
                    for (int k = 0; k < nb; ++k) {
                        double s = 0.0;
                        for (int j = 0; j < rb; ++j) s += left[i * rb + j] * B->transform[j * B->ncart + k];
                        cart[i * nb + k] = s;
                    }
            } else {
                memcpy(cart, left, sizeof(double) * (size_t)(na * nb));
            }
            int allzero = 1;
            for (int i = 0; i < na * nb; ++i) {
                if (a != bb) cart[i] *= 2.0;
                if (cart[i] != 0.0) allzero = 0;
            }
            if (allzero) continue;
            const int la = A->l, lb = B->l, L = la + lb;
            const int nlist = hermite_count(L);
            const double AB2 = sq_norm3(A->origin[0] - B->origin[0], A->origin[1] - B->origin[1],
                                        A->origin[2] - B->origin[2]);
            for (int p = 0; p < A->nprim; ++p)
                for (int q = 0; q < B->nprim; ++q) {
                    const double alpha = A->exps[p], beta = B->exps[q];
                    const double exponent = alpha + beta;
                    double center[3];
                    for (int c = 0; c < 3; ++c) center[c] = (alpha * A->origin[c] + beta * B->origin[c]) / exponent;
                    const double scale = exp(-alpha * beta / exponent * AB2) * 2.0 * KO_PI / exponent;
                    hermite_table(la, lb, exponent, center[0] - A->origin[0], center[0] - B->origin[0], ex);
                    hermite_table(la, lb, exponent, center[1] - A->origin[1], center[1] - B->origin[1], ey);
                    hermite_table(la, lb, exponent, center[2] - A->origin[2], center[2] - B->origin[2], ez);
                    for (int k = 0; k < nlist; ++k) pc[k] = 0.0;
                    const int width = L + 1;
                    for (int i = 0; i < na; ++i) {
                        const int* pi = A->powers[i];
                        for (int j = 0; j < nb; ++j) {
                            const int* pj = B->powers[j];
                            const double weight =
                                cart[i * nb + j] * A->weights[i * A->nprim + p] * B->weights[j * B->nprim + q];
                            if (weight == 0.0) continue;
                            for (int k = 0; k < nlist; ++k) {
                                const int* h = e->triples[k];
                                if (h[0] > pi[0] + pj[0] || h[1] > pi[1] + pj[1] || h[2] > pi[2] + pj[2]) continue;
                                pc[k] += weight * hget(ex, lb, width, pi[0], pj[0], h[0]) *
                                         hget(ey, lb, width, pi[1], pj[1], h[1]) *
                                         hget(ez, lb, width, pi[2], pj[2], h[2]);
                            }
                        }
                    }
                    int nz = 0;
                    for (int k = 0; k < nlist; ++k) nz |= pc[k] != 0.0;
                    if (!nz) continue;
                    if (e->npairs == e->cap_pairs) {
                        e->cap_pairs = e->cap_pairs ? 2 * e->cap_pairs : 1024;
                        e->pairs = (ko_pair*)realloc(e->pairs, sizeof(ko_pair) * (size_t)e->cap_pairs);
                    }
                    if (e->ncoef + nlist > e->cap_coef) {
                        e->cap_coef = (e->cap_coef ? 2 * e->cap_coef : 8192) + nlist;
                        e->coef = (double*)realloc(e->coef, sizeof(double) * (size_t)e->cap_coef);
                    }
                    ko_pair* pr = &e->pairs[e->npairs++];
                    pr->exponent = exponent;
                    memcpy(pr->center, center, sizeof center);
                    pr->order = L;
                    pr->first = e->ncoef;
                    for (int k = 0; k < nlist; ++k) e->coef[e->ncoef++] = scale * pc[k];
                }
        }
    }
    free(ex);
    free(ey);
    free(ez);
    free(pc);
    return e;
}

void ko_esp_destroy(ko_esp* e) {
    if (!e) return;
    free(e->pairs);
    free(e->coef);
    free(e->hidx);
    free(e->triples);
    free(e->xyz);
    free(e->charge);
    free(e);
}

long ko_esp_pair_count(const ko_esp* e) { return e->npairs; }

void ko_esp_nuclear(const ko_esp* e, const double* pts, long npts, double* out) {
    for (long j = 0; j < npts; ++j) {
        double sum = 0.0;
        for (int a = 0; a < e->natoms; ++a) {
            const double d = sqrt(sq_norm3(e->xyz[3 * a] - pts[3 * j], e->xyz[3 * a + 1] - pts[3 * j + 1],
                                           e->xyz[3 * a + 2] - pts[3 * j + 2]));
            if (e->charge[a] == 0.0 || d < 1e-8) continue;
            sum += e->charge[a] / d;
        }
        out[j] = sum;
    }
}

/* hermite_integrals + hermite_recursion + pair_potential,
 * src/electrostatic_potential.cpp:269-338 */
static double pair_potential(const ko_esp* e, const ko_pair* pr, const double* pt, double* prev,
                             double* cur) {
    const double pc[3] = {pr->center[0] - pt[0], pr->center[1] - pt[1], pr->center[2] - pt[2]};
    const int L = pr->order;
    double seeds[KO_BOYS_MAX + 1];
    ko_boys(pr->exponent * sq_norm3(pc[0], pc[1], pc[2]), L + 1, seeds);
    double power = 1.0;
    for (int k = 1; k <= L; ++k) {
        power *= -2.0 * pr->exponent;
        seeds[k] *= power;
    }
    const int side = e->side;
#define OFF(t, u, v) (((t) * side + (u)) * side + (v))
    for (int lev = L; lev >= 0; --lev) {
        double* t = prev;
        prev = cur;
        cur = t;
        cur[0] = seeds[lev];
        const int entries = hermite_count(L - lev);
        for (int k = 1; k < entries; ++k) {
            const int* h = e->triples[k];
            double value;
            if (h[0] > 0) {
                value = pc[0] * prev[OFF(h[0] - 1, h[1], h[2])];
                if (h[0] > 1) value += (h[0] - 1) * prev[OFF(h[0] - 2, h[1], h[2])];
            } else if (h[1] > 0) {
                value = pc[1] * prev[OFF(h[0], h[1] - 1, h[2])];
                if (h[1] > 1) value += (h[1] - 1) * prev[OFF(h[0], h[1] - 2, h[2])];
            } else {
                value = pc[2] * prev[OFF(h[0], h[1], h[2] - 1)];
                if (h[2] > 1) value += (h[2] - 1) * prev[OFF(h[0], h[1], h[2] - 2)];
            }
            cur[OFF(h[0], h[1], h[2])] = value;
        }
    }
#undef OFF
    const double* c = e->coef + pr->first;
    double sum = 0.0;
    const int nk = hermite_count(L);
    for (int k = 0; k < nk; ++k) sum += c[k] * cur[e->hidx[k]];
    return sum;
}

void ko_esp_evaluate(const ko_esp* e, const double* pts, long npts, double* out) {
    ko_esp_nuclear(e, pts, npts, out);
#pragma omp parallel
    {
        const long cube = (long)e->side * e->side * e->side;
        double* a = (double*)calloc((size_t)cube, sizeof(double));
        double* b = (double*)calloc((size_t)cube, sizeof(double));
#pragma omp for schedule(dynamic, 16)
        for (long j = 0; j < npts; ++j) {
            double sum = 0.0;
            for (long i = 0; i < e->npairs; ++i) {
                /* the recursion leaves R^0 in the buffer used last; pass the
                 * two buffers in a fixed order for every pair */
                sum += pair_potential(e, &e->pairs[i], pts + 3 * j, a, b);
            }
            out[j] = out[j] - sum;
        }
        free(a);
        free(b);
    }
}

void ko_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ko_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
