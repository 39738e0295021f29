/*
 * Parity oracle (test infrastructure only; see oracle.h).  Each function cites
 * the reference lines it restates.  Everything is scalar, FP64 and written
 * for clarity, not speed.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- Board symmetries (Board/BitBoard.cpp:4-84), square by square -------- */

static int square_after(int which, int b)
{
    int x = b & 7, y = b >> 3;
    switch (which) {
        case 0: return (7 - x) * 8 + (7 - y); /* codiagonal */
        case 1: return x * 8 + y;             /* diagonal */
        case 2: return y * 8 + (7 - x);       /* horizontal */
        default: return (7 - y) * 8 + x;      /* vertical */
    }
}

uint64_t or_flip(int which, uint64_t b)
{
    uint64_t r = 0;
    for (int s = 0; s < 64; s++)
        if ((b >> s) & 1) r |= 1ULL << square_after(which, s);
    return r;
}

typedef struct {
    uint64_t p, o;
} pos_t;

static pos_t flip_pos(int which, pos_t a)
{
    pos_t r = {or_flip(which, a.p), or_flip(which, a.o)};
    return r;
}
#define FC(x) flip_pos(0, x)
#define FD(x) flip_pos(1, x)
#define FH(x) flip_pos(2, x)
#define FV(x) flip_pos(3, x)

/* ---- FastIndex (Pattern/Helpers.cpp:5-47): PExt then the SumPow3 table ---- */

static uint64_t pext(uint64_t src, uint64_t mask)
{
    uint64_t r = 0;
    int i = 0;
    for (; mask; mask &= mask - 1, i++)
        if (src & mask & (0 - mask)) r |= 1ULL << i;
    return r;
}

static uint32_t sum_pow3(uint64_t bits)
{
    uint32_t sum = 0, w = 1;
    for (; bits; bits >>= 1, w *= 3)
        if (bits & 1) sum += w;
    return sum;
}

uint32_t or_fast_index(uint64_t p, uint64_t o, uint64_t mask)
{
    return sum_pow3(pext(p, mask)) + 2 * sum_pow3(pext(o, mask));
}

static uint32_t fi(pos_t a, uint64_t mask) { return or_fast_index(a.p, a.o, mask); }

static int popcount64(uint64_t x)
{
    int n = 0;
    for (; x; x &= x - 1) n++;
    return n;
}

static int pown3(int e)
{
    int r = 1;
    while (e-- > 0) r *= 3;
    return r;
}

/* ---- Indexers (Pattern/Indexer.cpp:17-365) ------------------------------- */

enum { K_A, K_V, K_D, K_VH, K_DC, K_VHDC };

typedef struct {
    int kind;
    uint64_t pattern;
    int order;
    int64_t space;
    uint32_t half_size, diag_size;
    uint32_t* dense;
} indexer_t;

static const uint64_t V_HALF = 0x00000000FFFFFFFFULL;
static const uint64_t D_HALF = 0x0080C0E0F0F8FCFEULL;
static const uint64_t D_DIAG = 0x8040201008040201ULL;

static uint64_t pdep(uint64_t src, uint64_t mask)
{
    uint64_t r = 0;
    for (int i = 0; mask; mask &= mask - 1, i++)
        if ((src >> i) & 1) r |= mask & (0 - mask);
    return r;
}

/* Dense orbit tables: Configurations order (Pattern/Helpers.cpp:81-102). */
static void build_dense(indexer_t* ix)
{
    uint64_t m = ix->pattern;
    int64_t n = pown3(popcount64(m));
    ix->dense = (uint32_t*)malloc(sizeof(uint32_t) * n);
    for (int64_t i = 0; i < n; i++) ix->dense[i] = 0xFFFFFFFFu;
    uint64_t size = 1ULL << popcount64(m);
    uint32_t index = 0;
    for (uint64_t p = 0; p < size; p++)
        for (uint64_t o = 0; o < size; o++) {
            if (p & o) continue;
            pos_t c = {pdep(p, m), pdep(o, m)};
            if (ix->dense[fi(c, m)] != 0xFFFFFFFFu) continue;
            pos_t v[8];
            int nv;
            if (ix->kind == K_VH) { /* :165-174 */
                v[0] = c; v[1] = FV(c); v[2] = FH(c); v[3] = FH(FV(c)); nv = 4;
            } else if (ix->kind == K_DC) { /* :219-228 */
                v[0] = c; v[1] = FD(c); v[2] = FC(c); v[3] = FC(FD(c)); nv = 4;
            } else { /* :273-290 */
                v[0] = c; v[1] = FC(c); v[2] = FD(c); v[3] = FH(c); v[4] = FV(c);
                v[5] = FC(FH(c)); v[6] = FD(FH(c)); v[7] = FV(FH(c)); nv = 8;
            }
            for (int i = 0; i < nv; i++) ix->dense[fi(v[i], m)] = index;
            index++;
        }
    ix->space = index;
}

static void make_indexer(uint64_t p, int mode, indexer_t* ix)
{
    memset(ix, 0, sizeof *ix);
    ix->pattern = p;
    if (mode == 1) {
        ix->kind = K_A;
        ix->order = 8;
        ix->space = pown3(popcount64(p));
        return;
    }
    /* CreateIndexer (:319-365) */
    int v = or_flip(3, p) == p, h = or_flip(2, p) == p, d = or_flip(1, p) == p, c = or_flip(0, p) == p;
    if (v && h && d && c) {
        ix->kind = K_VHDC; ix->order = 1; build_dense(ix);
    } else if (v && h) {
        ix->kind = K_VH; ix->order = 2; build_dense(ix);
    } else if (d && c) {
        ix->kind = K_DC; ix->order = 2; build_dense(ix);
    } else if (v || h) {
        ix->kind = K_V; ix->order = 4;
        if (!v) ix->pattern = or_flip(1, p);
        ix->half_size = (uint32_t)pown3(popcount64(ix->pattern & V_HALF));
        ix->space = (int64_t)ix->half_size * (ix->half_size + 1) / 2;
    } else if (d || c) {
        ix->kind = K_D; ix->order = 4;
        if (!d) ix->pattern = or_flip(3, p);
        ix->half_size = (uint32_t)pown3(popcount64(ix->pattern & D_HALF));
        ix->diag_size = (uint32_t)pown3(popcount64(ix->pattern & D_DIAG));
        ix->space = (int64_t)ix->diag_size * ix->half_size * (ix->half_size + 1) / 2;
    } else {
        ix->kind = K_A; ix->order = 8; ix->space = pown3(popcount64(p));
    }
}

static uint32_t index_of(const indexer_t* ix, pos_t a)
{
    uint64_t m = ix->pattern;
    switch (ix->kind) {
        case K_A: return fi(a, m); /* :27-30 */
        case K_V: { /* :74-81 */
            uint32_t mn = fi(a, m & V_HALF), mx = fi(FV(a), m & V_HALF);
            if (mn > mx) { uint32_t t = mn; mn = mx; mx = t; }
            return mn * ix->half_size + mx - (mn * (mn + 1) / 2);
        }
        case K_D: { /* :118-126 */
            uint32_t dd = fi(a, m & D_DIAG);
            uint32_t mn = fi(a, m & D_HALF), mx = fi(FD(a), m & D_HALF);
            if (mn > mx) { uint32_t t = mn; mn = mx; mx = t; }
            return (mn * ix->half_size + mx - (mn * (mn + 1) / 2)) * ix->diag_size + dd;
        }
        default: return ix->dense[fi(a, m)];
    }
}

static int insert_indices(const indexer_t* ix, pos_t a, uint32_t* loc, uint32_t off)
{
    switch (ix->kind) {
        case K_A: /* :32-41 */
            loc[0] = off + index_of(ix, a);
            loc[1] = off + index_of(ix, FC(a));
            loc[2] = off + index_of(ix, FD(a));
            loc[3] = off + index_of(ix, FH(a));
            loc[4] = off + index_of(ix, FV(a));
            loc[5] = off + index_of(ix, FH(FC(a)));
            loc[6] = off + index_of(ix, FH(FD(a)));
            loc[7] = off + index_of(ix, FH(FV(a)));
            return 8;
        case K_V: /* :83-89 */
            loc[0] = off + index_of(ix, a);
            loc[1] = off + index_of(ix, FC(a));
            loc[2] = off + index_of(ix, FD(a));
            loc[3] = off + index_of(ix, FH(a));
            return 4;
        case K_D: /* :128-134 */
            loc[0] = off + index_of(ix, a);
            loc[1] = off + index_of(ix, FC(a));
            loc[2] = off + index_of(ix, FH(a));
            loc[3] = off + index_of(ix, FV(a));
            return 4;
        case K_VH: /* :187-191 */
            loc[0] = off + index_of(ix, a);
            loc[1] = off + index_of(ix, FD(a));
            return 2;
        case K_DC: /* :241-245 */
            loc[0] = off + index_of(ix, a);
            loc[1] = off + index_of(ix, FV(a));
            return 2;
        default: /* :306-309 */
            loc[0] = off + index_of(ix, a);
            return 1;
    }
}

int or_group_info(const uint64_t* masks, int n, int mode, int64_t* cols, int* k)
{
    int64_t c = 0;
    int kk = 0;
    for (int i = 0; i < n; i++) {
        if (masks[i] == 0 || popcount64(masks[i]) > 16) return -1;
        indexer_t ix;
        make_indexer(masks[i], mode, &ix);
        c += ix.space;
        kk += ix.order;
        free(ix.dense);
    }
    *cols = c;
    *k = kk;
    return 0;
}

int or_group_index(const uint64_t* masks, int n, int mode, const uint64_t* po, int64_t rows, uint32_t* out)
{
    indexer_t* ix = (indexer_t*)calloc((size_t)n, sizeof(indexer_t));
    int k = 0;
    for (int i = 0; i < n; i++) {
        if (masks[i] == 0 || popcount64(masks[i]) > 16) {
            free(ix);
            return -1;
        }
        make_indexer(masks[i], mode, &ix[i]);
        k += ix[i].order;
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < rows; r++) {
        pos_t a = {po[2 * r], po[2 * r + 1]};
        uint32_t* loc = out + r * k;
        uint32_t off = 0; /* GroupIndexer::InsertIndices (:413-422) */
        for (int i = 0; i < n; i++) {
            loc += insert_indices(&ix[i], a, loc, off);
            off += (uint32_t)ix[i].space;
        }
    }
    for (int i = 0; i < n; i++) free(ix[i].dense);
    free(ix);
    return 0;
}

/* ---- MatrixCSR products (Math/MatrixCSR.cpp:21-87), FP64 ----------------- */

void or_spmv(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* x, double* y)
{
    (void)cols;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < rows; r++) {
        double s = 0;
        for (int j = 0; j < k; j++) s += x[idx[r * k + j]];
        y[r] = s;
    }
}

void or_spmv_t(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* y, double* x)
{
    memset(x, 0, sizeof(double) * (size_t)cols);
    for (int64_t r = 0; r < rows; r++)
        for (int j = 0; j < k; j++) x[idx[r * k + j]] += y[r];
}

static int cmp_u32(const void* a, const void* b)
{
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : x > y;
}

void or_jacobi(int k, int64_t rows, int64_t cols, const uint32_t* idx, double* d)
{
    double* diag = (double*)calloc((size_t)cols, sizeof(double));
    uint32_t* row = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)k);
    for (int64_t r = 0; r < rows; r++) {
        memcpy(row, idx + r * k, sizeof(uint32_t) * (size_t)k);
        qsort(row, (size_t)k, sizeof(uint32_t), cmp_u32);
        for (int i = 0, j; i < k; i = j) { /* duplicates count m^2 (:34-40) */
            j = i + 1;
            while (j < k && row[i] == row[j]) j++;
            diag[row[i]] += (double)(j - i) * (j - i);
        }
    }
    for (int64_t c = 0; c < cols; c++) d[c] = 1.0 / diag[c]; /* inv() (Math/Vector.cpp:117-124) */
    free(row);
    free(diag);
}

static double dot(const double* a, const double* b, int64_t n)
{
    double s = 0;
    for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

double or_normal_residual(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, const double* x)
{
    double* ax = (double*)malloc(sizeof(double) * (size_t)(rows ? rows : 1));
    double* g = (double*)malloc(sizeof(double) * (size_t)(cols ? cols : 1));
    or_spmv_t(k, rows, cols, idx, b, g);
    double bn = sqrt(dot(g, g, cols));
    or_spmv(k, rows, cols, idx, x, ax);
    for (int64_t r = 0; r < rows; r++) ax[r] = b[r] - ax[r];
    or_spmv_t(k, rows, cols, idx, ax, g);
    double rn = sqrt(dot(g, g, cols));
    free(ax);
    free(g);
    return bn > 0 ? rn / bn : rn;
}

/* A'A v through the two products (TwoMatrix, Math/MatrixProxy.h:63-67). */
static void normal_apply(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* v, double* tmp,
                         double* out)
{
    or_spmv(k, rows, cols, idx, v, tmp);
    or_spmv_t(k, rows, cols, idx, tmp, out);
}

int or_pcg(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int jacobi, int iterations,
           double tol, int check_every, double* x, double* residuum)
{
    size_t cb = sizeof(double) * (size_t)(cols ? cols : 1);
    double *P = malloc(cb), *r = malloc(cb), *z = malloc(cb), *p = malloc(cb), *Ap = malloc(cb);
    double* tmp = malloc(sizeof(double) * (size_t)(rows ? rows : 1));
    /* DiagonalPreconditioner(JacobiPreconditionerOfATA(A)) (Math/Solver.h:25-38) */
    if (jacobi) {
        or_jacobi(k, rows, cols, idx, P);
        for (int64_t c = 0; c < cols; c++)
            if (!isnormal(P[c])) P[c] = 1;
    } else {
        for (int64_t c = 0; c < cols; c++) P[c] = 1;
    }
    /* PCG(transposed(A) * A, P, 0, transposed(A) * b) (PatternFit/PatternFit.cpp:31, Math/Solver.h:88-97) */
    memset(x, 0, cb);
    or_spmv_t(k, rows, cols, idx, b, r); /* r = b' - A'A x0 with x0 = 0 */
    for (int64_t c = 0; c < cols; c++) p[c] = z[c] = P[c] * r[c];
    int it = 0;
    if (check_every <= 0) check_every = 1;
    for (; it < iterations;) { /* Iterate (:99-112) */
        double rz_old = dot(r, z, cols);
        normal_apply(k, rows, cols, idx, p, tmp, Ap);
        double pap = dot(p, Ap, cols);
        if (pap == 0) break;
        double alpha = rz_old / pap;
        for (int64_t c = 0; c < cols; c++) x[c] += alpha * p[c];
        for (int64_t c = 0; c < cols; c++) r[c] -= alpha * Ap[c];
        for (int64_t c = 0; c < cols; c++) z[c] = P[c] * r[c];
        double beta = dot(r, z, cols) / rz_old;
        for (int64_t c = 0; c < cols; c++) p[c] = z[c] + beta * p[c];
        it++;
        if (tol > 0 && it % check_every == 0 && or_normal_residual(k, rows, cols, idx, b, x) <= tol) break;
    }
    *residuum = dot(r, r, cols); /* Residuum (:114) */
    free(P); free(r); free(z); free(p); free(Ap); free(tmp);
    return it;
}

/* decompose (Math/Solver.h:119-126) */
static double decompose(double* v, int64_t n)
{
    double len = sqrt(dot(v, v, n));
    if (len == 0) return 0;
    for (int64_t i = 0; i < n; i++) v[i] /= len;
    return len;
}

/* Column scale of LSQR/LSMR on A S: s_c = diag(A'A)_c^-1/2, 1 for an empty
 * column (returns NULL when scale == 0: the reference's unscaled methods).
 * Column scaling is the diagonal right preconditioning that Paige and
 * Saunders (1982, section 5.4) recommend for LSQR; the reference has none. */
static double* column_scale(int scale, int k, int64_t rows, int64_t cols, const uint32_t* idx)
{
    if (!scale) return NULL;
    double* s = malloc(sizeof(double) * (size_t)(cols ? cols : 1));
    or_jacobi(k, rows, cols, idx, s); /* 1/diag, inf for an empty column */
    for (int64_t c = 0; c < cols; c++) s[c] = isfinite(s[c]) && s[c] > 0 ? sqrt(s[c]) : 1.0;
    return s;
}

/* y = A (S v) and v = S (A' y) */
static void spmv_s(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* s, const double* v,
                   double* tmp, double* y)
{
    if (!s) { or_spmv(k, rows, cols, idx, v, y); return; }
    for (int64_t c = 0; c < cols; c++) tmp[c] = s[c] * v[c];
    or_spmv(k, rows, cols, idx, tmp, y);
}
static void spmv_t_s(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* s, const double* y,
                     double* v)
{
    or_spmv_t(k, rows, cols, idx, y, v);
    if (s) for (int64_t c = 0; c < cols; c++) v[c] *= s[c];
}

int or_lsqr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int iterations, double tol,
            int check_every, double* x, double* residuum)
{
    return or_lsqr_scaled(k, rows, cols, idx, b, 0, iterations, tol, check_every, x, residuum);
}

int or_lsqr_scaled(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int scale,
                   int iterations, double tol, int check_every, double* x, double* residuum)
{
    size_t cb = sizeof(double) * (size_t)(cols ? cols : 1), rb = sizeof(double) * (size_t)(rows ? rows : 1);
    double *u = malloc(rb), *tu = malloc(rb), *v = malloc(cb), *tv = malloc(cb), *w = malloc(cb),
           *tmp = malloc(cb);
    double* sc = column_scale(scale, k, rows, cols, idx);
    memset(x, 0, cb);
    memcpy(u, b, rb); /* (:139-151) */
    double beta = decompose(u, rows);
    spmv_t_s(k, rows, cols, idx, sc, u, v);
    double alpha = decompose(v, cols);
    memcpy(w, v, cb);
    double phi_bar = beta, rho_bar = alpha;
    int it = 0;
    if (check_every <= 0) check_every = 1;
    for (; it < iterations;) { /* Iterate (:153-177) */
        spmv_s(k, rows, cols, idx, sc, v, tmp, tu);
        for (int64_t i = 0; i < rows; i++) u[i] = tu[i] - alpha * u[i];
        beta = decompose(u, rows);
        spmv_t_s(k, rows, cols, idx, sc, u, tv);
        for (int64_t i = 0; i < cols; i++) v[i] = tv[i] - beta * v[i];
        alpha = decompose(v, cols);
        double rho = sqrt(rho_bar * rho_bar + beta * beta);
        if (rho == 0) break;
        double c = rho_bar / rho, s = beta / rho;
        double theta = s * alpha;
        rho_bar = -c * alpha;
        double phi = c * phi_bar;
        phi_bar = s * phi_bar;
        for (int64_t i = 0; i < cols; i++) x[i] += (phi / rho) * (sc ? sc[i] : 1.0) * w[i];
        for (int64_t i = 0; i < cols; i++) w[i] = v[i] - (theta / rho) * w[i];
        it++;
        if (tol > 0 && it % check_every == 0 && or_normal_residual(k, rows, cols, idx, b, x) <= tol) break;
    }
    *residuum = phi_bar; /* Residuum (:179) */
    free(u); free(tu); free(v); free(tv); free(w); free(tmp); free(sc);
    return it;
}

/* signum and GivensRotation (Math/Solver.h:184-220: the scipy lsqr.py
 * sym_ortho form): c, s, r with c*a + s*b = r, signs as there. */
static double or_signum(double v) { return v < 0 ? -1.0 : (v > 0 ? 1.0 : 0.0); }
static void or_givens(double a, double b, double* c, double* s, double* r)
{
    if (b == 0) { *c = or_signum(a); *s = 0; *r = fabs(a); return; }
    if (a == 0) { *c = 0; *s = or_signum(b); *r = fabs(b); return; }
    if (fabs(b) > fabs(a)) {
        double tau = a / b;
        *s = or_signum(b) / sqrt(1 + tau * tau);
        *c = *s * tau;
        *r = b / *s;
    } else {
        double tau = b / a;
        *c = or_signum(a) / sqrt(1 + tau * tau);
        *s = *c * tau;
        *r = a / *c;
    }
}

/* LSMR (Math/Solver.h:222-287) from x0 = 0, FP64.  Writes x and |zeta_bar|
 * (the LSMR estimate of ||A'r||; the reference's Residuum() returns 0). */
int or_lsmr(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int iterations, double tol,
            int check_every, double* x, double* zeta_bar_out)
{
    return or_lsmr_scaled(k, rows, cols, idx, b, 0, iterations, tol, check_every, x, zeta_bar_out);
}

int or_lsmr_scaled(int k, int64_t rows, int64_t cols, const uint32_t* idx, const double* b, int scale,
                   int iterations, double tol, int check_every, double* x, double* zeta_bar_out)
{
    size_t cb = sizeof(double) * (size_t)(cols ? cols : 1), rb = sizeof(double) * (size_t)(rows ? rows : 1);
    double *u = malloc(rb), *tu = malloc(rb), *v = malloc(cb), *tv = malloc(cb), *h = malloc(cb),
           *hb = malloc(cb), *tmp = malloc(cb);
    double* sc = column_scale(scale, k, rows, cols, idx);
    memset(x, 0, cb);
    memcpy(u, b, rb); /* constructor (:236-251) */
    double beta = decompose(u, rows);
    spmv_t_s(k, rows, cols, idx, sc, u, v);
    double alpha = decompose(v, cols);
    double alpha_bar = alpha, zeta_bar = alpha * beta, rho = 1, rho_bar = 1, c_bar = 1, s_bar = 0;
    memcpy(h, v, cb);
    memset(hb, 0, cb);
    int it = 0;
    if (check_every <= 0) check_every = 1;
    for (; it < iterations;) { /* Iterate (:253-282) */
        double rho_old = rho, rho_bar_old = rho_bar;
        spmv_s(k, rows, cols, idx, sc, v, tmp, tu);
        for (int64_t i = 0; i < rows; i++) u[i] = tu[i] - alpha * u[i];
        beta = decompose(u, rows);
        spmv_t_s(k, rows, cols, idx, sc, u, tv);
        for (int64_t i = 0; i < cols; i++) v[i] = tv[i] - beta * v[i];
        alpha = decompose(v, cols);
        double c_hat, s_hat, alpha_hat;
        or_givens(alpha_bar, 0, &c_hat, &s_hat, &alpha_hat);
        double c, s;
        or_givens(alpha_hat, beta, &c, &s, &rho);
        double theta_new = s * alpha;
        alpha_bar = c * alpha;
        double theta_bar = s_bar * rho;
        double cb_in = c_bar * rho;
        or_givens(cb_in, theta_new, &c_bar, &s_bar, &rho_bar);
        double zeta = c_bar * zeta_bar;
        zeta_bar *= -s_bar;
        double f_hb = theta_bar * rho / rho_old / rho_bar_old, f_x = zeta / rho / rho_bar, f_h = theta_new / rho;
        for (int64_t i = 0; i < cols; i++) {
            hb[i] = h[i] - f_hb * hb[i];
            x[i] += f_x * (sc ? sc[i] : 1.0) * hb[i];
            h[i] = v[i] - f_h * h[i];
        }
        it++;
        if (tol > 0 && it % check_every == 0 && or_normal_residual(k, rows, cols, idx, b, x) <= tol) break;
    }
    *zeta_bar_out = fabs(zeta_bar);
    free(u); free(tu); free(v); free(tv); free(h); free(hb); free(tmp); free(sc);
    return it;
}

/* ------------------------------------------------------------------------
 * The seeded synthetic inputs of the tests and the benchmark, restated so
 * that a process that must not load the CUDA library (the benchmark's
 * reference arm) builds exactly the system the library's generator builds.
 * Random play follows RandomPlayer (Game/Player.cpp:3-16): a uniform choice
 * among the legal moves, a pass when the side to move has none; games that
 * end before the target empty count are replayed with the stream going on.
 * The stream is SplitMix64 (Steele, Lea and Flood 2014) used as a counter-
 * based generator: state seeded from (seed, index), advanced by the
 * golden-ratio increment and mixed on output.
 * ---------------------------------------------------------------------- */
static uint64_t sm_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
typedef struct { uint64_t s; } stream_t;
static stream_t sm_stream(uint64_t seed, uint64_t index)
{
    stream_t t = {sm_mix(seed ^ sm_mix(index + 0x632BE59BD9B4E019ULL))};
    return t;
}
static uint64_t sm_next(stream_t* t)
{
    t->s += 0x9E3779B97F4A7C15ULL;
    return sm_mix(t->s);
}
/* uniform in [0, n): multiply-high on 32 random bits */
static uint32_t sm_below(stream_t* t, uint32_t n) { return (uint32_t)(((sm_next(t) >> 32) * n) >> 32); }
/* uniform in (0, 1) */
static double sm_unit(stream_t* t) { return ((double)(sm_next(t) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

/* one square step in direction d of the 8 (bit 63 = A1, x = bit & 7) */
static uint64_t dir_step(uint64_t b, int d)
{
    switch (d) {
        case 0: return (b << 1) & 0xFEFEFEFEFEFEFEFEULL;
        case 1: return (b >> 1) & 0x7F7F7F7F7F7F7F7FULL;
        case 2: return b << 8;
        case 3: return b >> 8;
        case 4: return (b << 9) & 0xFEFEFEFEFEFEFEFEULL;
        case 5: return (b << 7) & 0x7F7F7F7F7F7F7F7FULL;
        case 6: return (b >> 7) & 0xFEFEFEFEFEFEFEFEULL;
        default: return (b >> 9) & 0x7F7F7F7F7F7F7F7FULL;
    }
}
static uint64_t moves_of(uint64_t p, uint64_t o)
{
    uint64_t m = 0;
    for (int d = 0; d < 8; d++) {
        uint64_t t = dir_step(p, d) & o;
        for (int i = 0; i < 5; i++) t |= dir_step(t, d) & o;
        m |= dir_step(t, d);
    }
    return m & ~(p | o);
}
static uint64_t flips_of(uint64_t p, uint64_t o, int sq)
{
    uint64_t all = 0;
    for (int d = 0; d < 8; d++) {
        uint64_t line = 0, x = dir_step(1ULL << sq, d);
        while (x & o) { line |= x; x = dir_step(x, d); }
        if (x & p) all |= line;
    }
    return all;
}

static int random_play(uint64_t seed, uint64_t i, int min_e, int max_e, uint64_t* out_p, uint64_t* out_o)
{
    stream_t rng = sm_stream(seed, i);
    const int target = min_e + (int)sm_below(&rng, (uint32_t)(max_e - min_e + 1));
    for (int attempt = 0; attempt < (1 << 16); attempt++) {
        uint64_t p = 0x0000000810000000ULL, o = 0x0000001008000000ULL; /* Position::Start() */
        int empties = 60, ended = 0;
        while (empties > target) {
            uint64_t m = moves_of(p, o);
            if (!m) {
                if (!moves_of(o, p)) { ended = 1; break; }
                uint64_t t = p; p = o; o = t; /* pass */
                continue;
            }
            uint32_t k = sm_below(&rng, (uint32_t)popcount64(m));
            while (k--) m &= m - 1;
            int sq = __builtin_ctzll(m);
            uint64_t f = flips_of(p, o, sq);
            uint64_t np = o ^ f;
            o = p ^ f ^ (1ULL << sq);
            p = np;
            empties--;
        }
        if (!ended) { *out_p = p; *out_o = o; return 1; }
    }
    *out_p = 0x0000000810000000ULL;
    *out_o = 0x0000001008000000ULL;
    return 0;
}

int or_generate_positions(uint64_t seed, int64_t first, int64_t n, int min_e, int max_e, uint64_t* po)
{
    if (n < 0 || first < 0 || min_e < 0 || min_e > max_e || max_e > 60) return -1;
    int ok = 1;
#pragma omp parallel for schedule(static) reduction(&& : ok)
    for (int64_t i = 0; i < n; i++) ok = random_play(seed, (uint64_t)(first + i), min_e, max_e, po + 2 * i, po + 2 * i + 1) && ok;
    return ok ? 0 : -1;
}

void or_generate_targets(int k, int64_t rows, int64_t cols, const uint32_t* idx, uint64_t seed, double w_sigma,
                         double noise_sigma, double* b, double* w_true)
{
    const double two_pi = 6.283185307179586;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < cols; c++) { /* w*_c ~ N(0, sigma^2), Box-Muller */
        stream_t t = sm_stream(seed ^ 0x5EED0F3EC7ED1ULL, (uint64_t)c);
        double u1 = sm_unit(&t), u2 = sm_unit(&t);
        w_true[c] = w_sigma * sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
    }
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < rows; r++) { /* b_r = clamp(2 rint(((A w*)_r + e_r) / 2), -64, 64) */
        double aw = 0;
        for (int j = 0; j < k; j++) aw += w_true[idx[r * k + j]];
        stream_t t = sm_stream(seed ^ 0xB0A5EDD15EA5EULL, (uint64_t)r);
        double u1 = sm_unit(&t), u2 = sm_unit(&t);
        double e = noise_sigma * sqrt(-2.0 * log(u1)) * cos(two_pi * u2);
        b[r] = fmin(64.0, fmax(-64.0, 2.0 * rint((aw + e) * 0.5)));
    }
}
