/*
 * Test infrastructure (oracle) -- NOT part of the product.
 *
 * A plain-C, long-double restatement of PFSOFTlib's forward DSOFT and inverse iDSOFT, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker. The CUDA
 * product never links, loads or calls this file.
 *
 * What it restates (paths relative to the reference project root):
 *   oracle_quadrature_weights  include/PFSOFTlib_headers/fn_dwt.hpp:62-83
 *   oracle_wigner_d            include/PFSOFTlib_headers/fn_dwt.hpp:105-200 (weighted) and
 *                              :237-332 (plain); seed :116-163, recurrence :167-199
 *   oracle_fft2_layers         src/fftw_wrapper.cpp:47-173 (FFTW_FORWARD = exp(-i..),
 *                              FFTW_BACKWARD = exp(+i..), unnormalised, per layer)
 *   oracle_dsoft               src/fn_dsoft.cpp:76-285
 *   oracle_idsoft              src/fn_idsoft.cpp:72-290
 *
 * The reference walks the order pairs (M, M') with M >= M' >= 0 and serves up to eight
 * coefficient columns from one Wigner matrix through fliplr/flipud and sign flips
 * (src/fn_dsoft.cpp:137-283, include/PFSOFTlib_headers/fn_flip.hpp:44-305). Written out, every
 * one of those cases follows one rule, which this file applies per coefficient (m1, m2):
 *   class      M = max(|m1|,|m2|), M' = min(|m1|,|m2|), d = the reference matrix for (M, M')
 *   position   FFT bin row = m2 mod N, col = m1 mod N of the layer-wise 2D DFT
 *   reversal   rev = (m1 < 0) xor (m2 < 0): beta_k is read as beta_{N-1-k} (pi - beta)
 *   sign       -1, times (-1)^(M-M') when x, times (-1)^(l-M) when rev, where
 *              x = (m1 < 0) if |m1| == M else (m2 > 0)
 *   forward    f^l_{m1,m2} = pi/(2B^2) * sign(l) * sum_k d[l][rev ? N-1-k : k] * F[k][col][row]
 *   inverse    H[k][col][row] = sum_l d'[l][rev ? N-1-k : k] * sign(l) * (2B^2/pi) * f^l_{m1,m2}
 * with d the weighted matrix (forward) and d' the unweighted one (inverse), both carrying the
 * reference's seed sign of -1 (fn_dwt.hpp:124-125 always evaluate to -1). The inverse writes
 * zero at the Nyquist bins row = B or col = B, which the reference leaves untouched
 * (they are zero when the caller passes a fresh grid).
 *
 * Arithmetic: weights, Wigner recurrence, FFT and the DWT sums in long double; inputs and
 * outputs are double.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef long double ld;
typedef long double complex ldc;

static const ld PI_L = 3.141592653589793238462643383279502884L;

size_t oracle_coef_offset(int l) { return (size_t)l * (4 * (size_t)l * l - 1) / 3; }

size_t oracle_coef_count(int B) { return oracle_coef_offset(B); }

/* packed index of f^l_{m1,m2}: column-major (2l+1)^2 block, negative orders wrapped
 * (src/dsoft_fourier_coefficients.cpp:80-89) */
size_t oracle_coef_index(int l, int m1, int m2)
{
    const size_t L = 2 * (size_t)l + 1;
    const size_t i1 = m1 >= 0 ? (size_t)m1 : L + m1;
    const size_t i2 = m2 >= 0 ? (size_t)m2 : L + m2;
    return oracle_coef_offset(l) + i2 * L + i1;
}

/* fn_dwt.hpp:62-83 */
void oracle_quadrature_weights_ld(int B, ld* w)
{
    for (int i = 0; i < B; ++i) {
        ld wi = 2.0L / B * sinl(PI_L * (2.0L * i + 1.0L) / (4.0L * B));
        ld sum = 0;
        for (int k = 0; k < B; ++k)
            sum += 1.0L / (2.0L * k + 1.0L) * sinl((2.0L * i + 1.0L) * (2.0L * k + 1.0L) * PI_L / (4.0L * B));
        wi *= sum;
        w[i] = wi;
        w[2 * B - 1 - i] = wi;
    }
}

void oracle_quadrature_weights(int B, double* w)
{
    ld* t = (ld*)malloc(sizeof(ld) * 2 * B);
    oracle_quadrature_weights_ld(B, t);
    for (int j = 0; j < 2 * B; ++j) w[j] = (double)t[j];
    free(t);
}

/* Rows l = J..B-1 of the reference Wigner d-matrix for orders (M, Mp), J = max(|M|,|Mp|),
 * written row-major out[(l-J)*2B + k] (fn_dwt.hpp:105-200, :237-332). w == NULL gives the
 * unweighted matrix. */
void oracle_wigner_d_ld(int B, int M, int Mp, const ld* w, ld* out)
{
    const int N = 2 * B;
    const int aM = abs(M), aMp = abs(Mp);
    const int J = aM > aMp ? aM : aMp;
    const int Jmin = aM < aMp ? aM : aMp;
    ld norm = sqrtl((2.0L * J + 1.0L) / 2.0L);
    for (int i = 0; i < J - Jmin; ++i) norm *= sqrtl((2.0L * J - i) / (i + 1.0L));
    /* fn_dwt.hpp:124-125: the two assignments leave the seed sign at -1 for every (M, Mp) */
    const ld seed_sign = -1.0L;
    int cp, sp; /* fn_dwt.hpp:128-148 */
    if (J == aM && M >= 0) { cp = J + Mp; sp = J - Mp; }
    else if (J == aM)      { cp = J - Mp; sp = J + Mp; }
    else if (Mp >= 0)      { cp = J + M;  sp = J - M;  }
    else                   { cp = J - M;  sp = J + M;  }
    ld* cb = (ld*)malloc(sizeof(ld) * N);
    for (int k = 0; k < N; ++k) {
        const ld beta = (2.0L * k + 1.0L) * PI_L / (4.0L * B);
        cb[k] = cosl(beta);
        ld v = norm * seed_sign * powl(sinl(0.5L * beta), sp) * powl(cosl(0.5L * beta), cp);
        out[k] = w ? v * w[k] : v;
    }
    for (int i = 0; i < B - J - 1; ++i) {
        const ld idx = (ld)(J + i);
        const ld nrm = sqrtl((2.0L * idx + 3.0L) / (2.0L * idx + 1.0L));
        const ld nom = (idx + 1.0L) * (2.0L * idx + 1.0L);
        const ld den = 1.0L / sqrtl(((idx + 1) * (idx + 1) - (ld)M * M) * ((idx + 1) * (idx + 1) - (ld)Mp * Mp));
        const ld f1 = nrm * nom * den;
        ld c1 = 0, f2 = 0;
        if (J + i != 0) {
            const ld t1 = sqrtl((2.0L * idx + 3.0L) / (2.0L * idx - 1.0L)) * (idx + 1.0L) / idx;
            const ld t2 = sqrtl((idx * idx - (ld)M * M) * (idx * idx - (ld)Mp * Mp));
            c1 = -t1 * t2 * den;
            f2 = -(ld)M * Mp / (idx * (idx + 1.0L));
        }
        const ld* cur = out + (size_t)i * N;
        const ld* prev = i ? out + (size_t)(i - 1) * N : NULL;
        ld* nxt = out + (size_t)(i + 1) * N;
        for (int k = 0; k < N; ++k) nxt[k] = c1 * (prev ? prev[k] : 0.0L) + cur[k] * f1 * (f2 + cb[k]);
    }
    free(cb);
}

void oracle_wigner_d(int B, int M, int Mp, int weighted, double* out)
{
    const int N = 2 * B;
    const int J = abs(M) > abs(Mp) ? abs(M) : abs(Mp);
    ld* w = NULL;
    if (weighted) { w = (ld*)malloc(sizeof(ld) * N); oracle_quadrature_weights_ld(B, w); }
    ld* d = (ld*)malloc(sizeof(ld) * (size_t)(B - J) * N);
    oracle_wigner_d_ld(B, M, Mp, w, d);
    for (size_t i = 0; i < (size_t)(B - J) * N; ++i) out[i] = (double)d[i];
    free(d);
    free(w);
}

/* ---- long-double mixed-radix FFT (Stockham autosort) with precomputed tables ---- */
typedef struct {
    int n, nst;
    int radix[64], ns[64];
    ldc* tw[64];    /* tw[s][k*R + r] = w^(r k), w = exp(sign 2 pi i/(ns R)) */
    ldc* rt[64];    /* rt[s][q*R + r] = exp(sign 2 pi i r q / R) */
} fft_plan_ld;

static ldc unit_root_ld(long long num, long long den, int sign)
{
    long long m = num % den;
    if (m < 0) m += den;
    const ld a = 2.0L * PI_L * (ld)m / (ld)den;
    return cosl(a) + I * (sign * sinl(a));
}

static void fft_plan_make(fft_plan_ld* p, int n, int sign)
{
    p->n = n;
    p->nst = 0;
    int rem = n, ns = 1;
    while (rem > 1) {
        int R = 0;
        if (rem % 4 == 0) R = 4;
        else if (rem % 2 == 0) R = 2;
        else for (int q = 3; q <= rem; q += 2) if (rem % q == 0) { R = q; break; }
        const int s = p->nst++;
        p->radix[s] = R;
        p->ns[s] = ns;
        p->tw[s] = (ldc*)malloc(sizeof(ldc) * (size_t)ns * R);
        p->rt[s] = (ldc*)malloc(sizeof(ldc) * (size_t)R * R);
        for (int k = 0; k < ns; ++k)
            for (int r = 0; r < R; ++r) p->tw[s][(size_t)k * R + r] = unit_root_ld((long long)r * k, (long long)ns * R, sign);
        for (int q = 0; q < R; ++q)
            for (int r = 0; r < R; ++r) p->rt[s][(size_t)q * R + r] = unit_root_ld((long long)r * q, R, sign);
        ns *= R;
        rem /= R;
    }
}

static void fft_plan_free(fft_plan_ld* p)
{
    for (int s = 0; s < p->nst; ++s) { free(p->tw[s]); free(p->rt[s]); }
}

static void fft1_ld(const fft_plan_ld* p, ldc* x, ldc* tmp, ldc* v)
{
    const int n = p->n;
    ldc* a = x;
    ldc* b = tmp;
    for (int s = 0; s < p->nst; ++s) {
        const int R = p->radix[s], ns = p->ns[s], m = n / R;
        for (int j = 0; j < m; ++j) {
            const int k = j % ns;
            const ldc* tw = p->tw[s] + (size_t)k * R;
            for (int r = 0; r < R; ++r) v[r] = a[j + r * m] * tw[r];
            const int ob = (j / ns) * ns * R + k;
            for (int q = 0; q < R; ++q) {
                const ldc* rt = p->rt[s] + (size_t)q * R;
                ldc acc = 0;
                for (int r = 0; r < R; ++r) acc += v[r] * rt[r];
                b[ob + q * ns] = acc;
            }
        }
        ldc* t = a; a = b; b = t;
    }
    if (a != x) memcpy(x, a, sizeof(ldc) * n);
}

/* Layer-wise unnormalised 2D DFT of an N x N x lays grid, rows contiguous
 * (fftw_wrapper.cpp:47-173). sign -1 = forward, +1 = inverse. */
void oracle_fft2_layers_ld(int N, int lays, ldc* g, int sign)
{
    fft_plan_ld plan;
    fft_plan_make(&plan, N, sign);
#pragma omp parallel
    {
        ldc* col = (ldc*)malloc(sizeof(ldc) * N);
        ldc* tmp = (ldc*)malloc(sizeof(ldc) * N);
        ldc* v = (ldc*)malloc(sizeof(ldc) * N);
#pragma omp for schedule(dynamic)
        for (int k = 0; k < lays; ++k) {
            ldc* L = g + (size_t)k * N * N;
            for (int c = 0; c < N; ++c) fft1_ld(&plan, L + (size_t)c * N, tmp, v);
            for (int r = 0; r < N; ++r) {
                for (int c = 0; c < N; ++c) col[c] = L[(size_t)c * N + r];
                fft1_ld(&plan, col, tmp, v);
                for (int c = 0; c < N; ++c) L[(size_t)c * N + r] = col[c];
            }
        }
        free(col);
        free(tmp);
        free(v);
    }
    fft_plan_free(&plan);
}

void oracle_fft2_layers(int N, int lays, const double* in, double* out, int sign)
{
    const size_t n = (size_t)N * N * lays;
    ldc* g = (ldc*)malloc(sizeof(ldc) * n);
    for (size_t i = 0; i < n; ++i) g[i] = in[2 * i] + I * in[2 * i + 1];
    oracle_fft2_layers_ld(N, lays, g, sign);
    for (size_t i = 0; i < n; ++i) { out[2 * i] = (double)creall(g[i]); out[2 * i + 1] = (double)cimagl(g[i]); }
    free(g);
}

/* The per-coefficient symmetry rule (see the header comment). */
static int case_rev(int m1, int m2) { return (m1 < 0) != (m2 < 0); }

static ld case_sign(int m1, int m2, int l)
{
    const int a1 = abs(m1), a2 = abs(m2);
    const int M = a1 > a2 ? a1 : a2, Mp = a1 < a2 ? a1 : a2;
    const int x = (a1 == M) ? (m1 < 0) : (m2 > 0);
    ld s = -1.0L;
    if (x && ((M - Mp) & 1)) s = -s;
    if (case_rev(m1, m2) && ((l - M) & 1)) s = -s;
    return s;
}

/* enumerate the distinct (m1, m2) served by class (M, Mp), M >= Mp >= 0 */
static int class_cases(int M, int Mp, int m1s[8], int m2s[8])
{
    int n = 0;
    const int c1[8] = {M, Mp, -M, -Mp, Mp, M, -Mp, -M};
    const int c2[8] = {Mp, M, -Mp, -M, -M, -Mp, M, Mp};
    for (int i = 0; i < 8; ++i) {
        int dup = 0;
        for (int j = 0; j < n; ++j) dup |= (m1s[j] == c1[i] && m2s[j] == c2[i]);
        if (!dup) { m1s[n] = c1[i]; m2s[n] = c2[i]; ++n; }
    }
    return n;
}

/* src/fn_dsoft.cpp:76-285. grid: N^3 complex (not modified); coeffs: packed B(4B^2-1)/3. */
void oracle_dsoft(const double* grid, int B, double* coeffs)
{
    const int N = 2 * B;
    const size_t n3 = (size_t)N * N * N;
    ldc* F = (ldc*)malloc(sizeof(ldc) * n3);
    for (size_t i = 0; i < n3; ++i) F[i] = grid[2 * i] + I * grid[2 * i + 1];
    oracle_fft2_layers_ld(N, N, F, -1);
    ld* w = (ld*)malloc(sizeof(ld) * N);
    oracle_quadrature_weights_ld(B, w);
    const ld norm = PI_L / ((ld)B * N);
    const int nclass = B * (B + 1) / 2;
#pragma omp parallel
    {
        ld* d = (ld*)malloc(sizeof(ld) * (size_t)B * N);
        ldc* s = (ldc*)malloc(sizeof(ldc) * N);
#pragma omp for schedule(dynamic)
        for (int c = 0; c < nclass; ++c) {
            int M = (int)((sqrt(8.0 * c + 1.0) - 1.0) / 2.0);
            while (M * (M + 1) / 2 > c) --M;
            while ((M + 1) * (M + 2) / 2 <= c) ++M;
            const int Mp = c - M * (M + 1) / 2;
            oracle_wigner_d_ld(B, M, Mp, w, d);
            int m1s[8], m2s[8];
            const int nc = class_cases(M, Mp, m1s, m2s);
            for (int q = 0; q < nc; ++q) {
                const int m1 = m1s[q], m2 = m2s[q];
                const int row = ((m2 % N) + N) % N, col = ((m1 % N) + N) % N;
                const int rev = case_rev(m1, m2);
                for (int k = 0; k < N; ++k) s[k] = F[((size_t)k * N + col) * N + row];
                for (int l = M; l < B; ++l) {
                    const ld* dl = d + (size_t)(l - M) * N;
                    ldc acc = 0;
                    for (int k = 0; k < N; ++k) acc += dl[rev ? N - 1 - k : k] * s[k];
                    acc *= norm * case_sign(m1, m2, l);
                    const size_t o = oracle_coef_index(l, m1, m2);
                    coeffs[2 * o] = (double)creall(acc);
                    coeffs[2 * o + 1] = (double)cimagl(acc);
                }
            }
        }
        free(d);
        free(s);
    }
    free(w);
    free(F);
}

/* src/fn_idsoft.cpp:72-290. coeffs: packed; grid: N^3 complex, fully overwritten. */
void oracle_idsoft(const double* coeffs, int B, double* grid)
{
    const int N = 2 * B;
    const size_t n3 = (size_t)N * N * N;
    ldc* H = (ldc*)calloc(n3, sizeof(ldc));
    const ld norm = (ld)B * N / PI_L;
    const int nclass = B * (B + 1) / 2;
#pragma omp parallel
    {
        ld* d = (ld*)malloc(sizeof(ld) * (size_t)B * N);
        ldc* g = (ldc*)malloc(sizeof(ldc) * B);
#pragma omp for schedule(dynamic)
        for (int c = 0; c < nclass; ++c) {
            int M = (int)((sqrt(8.0 * c + 1.0) - 1.0) / 2.0);
            while (M * (M + 1) / 2 > c) --M;
            while ((M + 1) * (M + 2) / 2 <= c) ++M;
            const int Mp = c - M * (M + 1) / 2;
            oracle_wigner_d_ld(B, M, Mp, NULL, d);
            int m1s[8], m2s[8];
            const int nc = class_cases(M, Mp, m1s, m2s);
            for (int q = 0; q < nc; ++q) {
                const int m1 = m1s[q], m2 = m2s[q];
                const int row = ((m2 % N) + N) % N, col = ((m1 % N) + N) % N;
                const int rev = case_rev(m1, m2);
                for (int l = M; l < B; ++l) {
                    const size_t o = oracle_coef_index(l, m1, m2);
                    g[l - M] = norm * case_sign(m1, m2, l) * (coeffs[2 * o] + I * (ld)coeffs[2 * o + 1]);
                }
                for (int k = 0; k < N; ++k) {
                    const int kk = rev ? N - 1 - k : k;
                    ldc acc = 0;
                    for (int l = M; l < B; ++l) acc += d[(size_t)(l - M) * N + kk] * g[l - M];
                    H[((size_t)k * N + col) * N + row] = acc;
                }
            }
        }
        free(d);
        free(g);
    }
    oracle_fft2_layers_ld(N, N, H, +1);
    const ld scale = 1.0L / (4.0L * B * B);
    for (size_t i = 0; i < n3; ++i) {
        grid[2 * i] = (double)(creall(H[i]) * scale);
        grid[2 * i + 1] = (double)(cimagl(H[i]) * scale);
    }
    free(H);
}

/* The discrete Wigner transform stage alone (fn_dsoft.cpp:134-283 / fn_idsoft.cpp:124-283), on
 * the engine's bin-major spectrum X[row][col][k] (the unnormalised layer-wise 2D DFT with beta
 * innermost), for a list of order classes only (indices in the M-major enumeration; NULL with
 * n < 0 = every class). Test infrastructure for the sharded transform, whose ranks each run the
 * DWT of their own classes. Forward: writes the classes' coefficients, scaled pi/(2B^2); every
 * other coefficient is left as it is. Inverse: writes the beta columns of the classes' bins,
 * scaled 2B^2/pi; every other value of X is left as it is. */
static void class_orders_ld(int c, int* M, int* Mp)
{
    int m = (int)((sqrt(8.0 * c + 1.0) - 1.0) / 2.0);
    while (m * (m + 1) / 2 > c) --m;
    while ((m + 1) * (m + 2) / 2 <= c) ++m;
    *M = m;
    *Mp = c - m * (m + 1) / 2;
}

void oracle_dwt_forward(const double* X, int B, const int* classes, int n, double* coeffs)
{
    const int N = 2 * B;
    const int count = n < 0 ? B * (B + 1) / 2 : n;
    ld* w = (ld*)malloc(sizeof(ld) * N);
    oracle_quadrature_weights_ld(B, w);
    const ld norm = PI_L / ((ld)B * N);
    ld* d = (ld*)malloc(sizeof(ld) * (size_t)B * N);
    for (int i = 0; i < count; ++i) {
        int M, Mp;
        class_orders_ld(n < 0 ? i : classes[i], &M, &Mp);
        oracle_wigner_d_ld(B, M, Mp, w, d);
        int m1s[8], m2s[8];
        const int nc = class_cases(M, Mp, m1s, m2s);
        for (int q = 0; q < nc; ++q) {
            const int m1 = m1s[q], m2 = m2s[q];
            const int row = ((m2 % N) + N) % N, col = ((m1 % N) + N) % N;
            const int rev = case_rev(m1, m2);
            const double* s = X + 2 * ((size_t)row * N + col) * N;
            for (int l = M; l < B; ++l) {
                const ld* dl = d + (size_t)(l - M) * N;
                ldc acc = 0;
                for (int k = 0; k < N; ++k) acc += dl[rev ? N - 1 - k : k] * (s[2 * k] + I * (ld)s[2 * k + 1]);
                acc *= norm * case_sign(m1, m2, l);
                const size_t o = oracle_coef_index(l, m1, m2);
                coeffs[2 * o] = (double)creall(acc);
                coeffs[2 * o + 1] = (double)cimagl(acc);
            }
        }
    }
    free(d);
    free(w);
}

void oracle_dwt_inverse(const double* coeffs, int B, const int* classes, int n, double* X)
{
    const int N = 2 * B;
    const int count = n < 0 ? B * (B + 1) / 2 : n;
    const ld norm = (ld)B * N / PI_L;
    ld* d = (ld*)malloc(sizeof(ld) * (size_t)B * N);
    ldc* g = (ldc*)malloc(sizeof(ldc) * B);
    for (int i = 0; i < count; ++i) {
        int M, Mp;
        class_orders_ld(n < 0 ? i : classes[i], &M, &Mp);
        oracle_wigner_d_ld(B, M, Mp, NULL, d);
        int m1s[8], m2s[8];
        const int nc = class_cases(M, Mp, m1s, m2s);
        for (int q = 0; q < nc; ++q) {
            const int m1 = m1s[q], m2 = m2s[q];
            const int row = ((m2 % N) + N) % N, col = ((m1 % N) + N) % N;
            const int rev = case_rev(m1, m2);
            for (int l = M; l < B; ++l) {
                const size_t o = oracle_coef_index(l, m1, m2);
                g[l - M] = norm * case_sign(m1, m2, l) * (coeffs[2 * o] + I * (ld)coeffs[2 * o + 1]);
            }
            double* s = X + 2 * ((size_t)row * N + col) * N;
            for (int k = 0; k < N; ++k) {
                const int kk = rev ? N - 1 - k : k;
                ldc acc = 0;
                for (int l = M; l < B; ++l) acc += d[(size_t)(l - M) * N + kk] * g[l - M];
                s[2 * k] = (double)creall(acc);
                s[2 * k + 1] = (double)cimagl(acc);
            }
        }
    }
    free(g);
    free(d);
}
