/* CPU oracle: plain-C restatement of the reference joint BP + PP decoder.
 * TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.
 * Pinned against the reference built from its own sources (oracle/_ref) by
 * tests/test_oracle_pin.py and by the golden fixtures under tests/golden/.
 * Every function cites the jointbp_ets.cpp lines whose behaviour it restates. */
#include "jbp_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int xbit(int s) { return (s == 1 || s == 3) ? 1 : 0; }   /* jointbp_ets.cpp:659-661 */
static int zbit(int s) { return (s == 2 || s == 3) ? 1 : 0; }   /* jointbp_ets.cpp:663-665 */
static int sbit(int side, int s) { return side == 0 ? xbit(s) : zbit(s); }

/* ---------------------------------------------------------------- code construction */

static long long mod_norm(long long x, long long m) { /* jointbp_ets.cpp:62-66 */
    long long r = x % m;
    return r < 0 ? r + m : r;
}

static long long egcd(long long a, long long b, long long *x, long long *y) { /* 68-78 */
    if (b == 0) { *x = 1; *y = 0; return a; }
    long long x1, y1;
    long long g = egcd(b, a % b, &x1, &y1);
    *x = y1;
    *y = x1 - (a / b) * y1;
    return g;
}

static int modinv(long long a, long long m, long long *inv) { /* 80-87 */
    a = mod_norm(a, m);
    if (m == 1) { *inv = 0; return 1; }
    long long x, y;
    if (egcd(a, m, &x, &y) != 1) return 0;
    *inv = mod_norm(x, m);
    return 1;
}

static int mod_index(int x, int m) { int r = x % m; return r < 0 ? r + m : r; }

static void csr_from_dense(int m, int deg, const int *dense, int **off, int **var, int *edges) {
    *off = (int *)malloc(sizeof(int) * (m + 1));
    *var = (int *)malloc(sizeof(int) * (size_t)m * deg);
    int k = 0;
    for (int c = 0; c < m; ++c) {
        (*off)[c] = k;
        for (int i = 0; i < deg; ++i) (*var)[k++] = dense[c * deg + i];
    }
    (*off)[m] = k;
    *edges = k;
}

/* Variable -> edge lists in ascending check order (build_var_adjacency, 922-935). */
static void build_var_side(jbo_code *c, int s) {
    int n = c->n, m = c->m[s];
    int *cnt = (int *)calloc(n + 1, sizeof(int));
    for (int e = 0; e < c->e[s]; ++e) cnt[c->chk_var[s][e] + 1]++;
    c->var_off[s] = (int *)malloc(sizeof(int) * (n + 1));
    c->var_off[s][0] = 0;
    for (int v = 0; v < n; ++v) c->var_off[s][v + 1] = c->var_off[s][v] + cnt[v + 1];
    c->var_edge[s] = (int *)malloc(sizeof(int) * (c->e[s] > 0 ? c->e[s] : 1));
    int *fill = (int *)calloc(n, sizeof(int));
    for (int ch = 0; ch < m; ++ch)
        for (int e = c->chk_off[s][ch]; e < c->chk_off[s][ch + 1]; ++e) {
            int v = c->chk_var[s][e];
            c->var_edge[s][c->var_off[s][v] + fill[v]++] = e;
        }
    free(cnt);
    free(fill);
}

/* Params file + APM blocks + check neighbours: read_params (162-180),
 * build_block_matrix_hx/hz (98-160), build_check_neighbors (628-648).
 * Codes with a missing block (non-invertible multiplier) are rejected: the reference
 * leaves -1 neighbours in that case and later indexes err[-1]. */
int jbo_code_from_params(const char *path, jbo_code *out) {
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "r");
    if (!f) return 1;
    long long P;
    int J, L;
    unsigned long long seed;
    if (fscanf(f, "%lld %d %d", &P, &J, &L) != 3 || fscanf(f, "%llu", &seed) != 1 || L % 2 != 0 || P <= 0 ||
        J <= 0 || L <= 0) {
        fclose(f);
        return 2;
    }
    int L2 = L / 2;
    long long *abcd = (long long *)malloc(sizeof(long long) * 4 * L2);
    for (int i = 0; i < 4 * L2; ++i)
        if (fscanf(f, "%lld", &abcd[i]) != 1) { fclose(f); free(abcd); return 2; }
    fclose(f);
    const long long *a = abcd, *b = abcd + L2, *cc = abcd + 2 * L2, *d = abcd + 3 * L2;
    int m = J * (int)P;
    int n = L * (int)P;
    int *dense = (int *)malloc(sizeof(int) * (size_t)m * L);
    int rc = 0;
    for (int side = 0; side < 2 && rc == 0; ++side) {
        for (int r = 0; r < J && rc == 0; ++r) {
            for (int col = 0; col < L; ++col) {
                long long A, B;
                if (side == 0) {
                    int idx = col < L2 ? mod_index(col - r, L2) : mod_index(col - L2 - r, L2);
                    A = mod_norm(col < L2 ? a[idx] : cc[idx], P);
                    B = mod_norm(col < L2 ? b[idx] : d[idx], P);
                } else {
                    int k = col < L2 ? mod_index(col - r, L2) : mod_index(col - L2 - r, L2);
                    int idx = mod_index(-k, L2);
                    long long inv;
                    long long mul = col < L2 ? cc[idx] : a[idx];
                    long long add = col < L2 ? d[idx] : b[idx];
                    if (!modinv(mod_norm(mul, P), P, &inv)) { rc = 3; break; }
                    A = inv;
                    B = mod_norm(-inv * mod_norm(add, P), P);
                }
                for (int x = 0; x < P; ++x) {
                    long long y = mod_norm(A * x + B, P);
                    dense[(size_t)(r * P + x) * L + col] = col * (int)P + (int)y;
                }
            }
        }
        if (rc == 0) {
            out->m[side] = m;
            csr_from_dense(m, L, dense, &out->chk_off[side], &out->chk_var[side], &out->e[side]);
        }
    }
    free(dense);
    free(abcd);
    if (rc) { jbo_code_free(out); return rc; }
    out->n = n;
    out->P = (int)P;
    build_var_side(out, 0);
    build_var_side(out, 1);
    return 0;
}

int jbo_code_from_checks(int n, int mx, const int *xoff, const int *xvar, int mz, const int *zoff,
                         const int *zvar, jbo_code *out) {
    memset(out, 0, sizeof(*out));
    out->n = n;
    const int *offs[2] = {xoff, zoff}, *vars[2] = {xvar, zvar};
    int ms[2] = {mx, mz};
    for (int s = 0; s < 2; ++s) {
        out->m[s] = ms[s];
        out->e[s] = offs[s][ms[s]];
        out->chk_off[s] = (int *)malloc(sizeof(int) * (ms[s] + 1));
        memcpy(out->chk_off[s], offs[s], sizeof(int) * (ms[s] + 1));
        out->chk_var[s] = (int *)malloc(sizeof(int) * (out->e[s] > 0 ? out->e[s] : 1));
        memcpy(out->chk_var[s], vars[s], sizeof(int) * out->e[s]);
        for (int e = 0; e < out->e[s]; ++e)
            if (vars[s][e] < 0 || vars[s][e] >= n) { jbo_code_free(out); return 1; }
        build_var_side(out, s);
    }
    return 0;
}

void jbo_code_free(jbo_code *c) {
    for (int s = 0; s < 2; ++s) {
        free(c->chk_off[s]); free(c->chk_var[s]); free(c->var_off[s]); free(c->var_edge[s]);
    }
    memset(c, 0, sizeof(*c));
}

/* compute_syndrome (1834-1849). */
void jbo_syndrome(const jbo_code *c, int side, const uint8_t *err, uint8_t *syn) {
    for (int ch = 0; ch < c->m[side]; ++ch) {
        int par = 0;
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) par ^= sbit(side, err[c->chk_var[side][e]]);
        syn[ch] = (uint8_t)par;
    }
}

static int syn_equal(const jbo_code *c, int side, const uint8_t *est, const uint8_t *target) {
    for (int ch = 0; ch < c->m[side]; ++ch) {
        int par = 0;
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) par ^= sbit(side, est[c->chk_var[side][e]]);
        if (par != target[ch]) return 0;
    }
    return 1;
}

static int unsat_count(const jbo_code *c, int side, const uint8_t *est, const uint8_t *target) {
    int k = 0;
    for (int ch = 0; ch < c->m[side]; ++ch) {
        int par = 0;
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) par ^= sbit(side, est[c->chk_var[side][e]]);
        k += (par != target[ch]);
    }
    return k;
}

/* ---------------------------------------------------------------- sampler */

/* splitmix64 finaliser and per-trial seed (4401-4411). */
static uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

uint64_t jbo_trial_seed(uint64_t base, uint64_t idx) { return splitmix64(base ^ (idx * 0x9e3779b97f4a7c15ull)); }

/* 64-bit Mersenne Twister (Matsumoto & Nishimura; the std::mt19937_64 parameters). */
typedef struct { uint64_t s[312]; int i; } mt64;

static void mt64_seed(mt64 *g, uint64_t seed) {
    g->s[0] = seed;
    for (int i = 1; i < 312; ++i) g->s[i] = 6364136223846793005ull * (g->s[i - 1] ^ (g->s[i - 1] >> 62)) + (uint64_t)i;
    g->i = 312;
}

static uint64_t mt64_next(mt64 *g) {
    if (g->i >= 312) {
        const uint64_t hi = 0xFFFFFFFF80000000ull, lo = 0x7FFFFFFFull;
        for (int k = 0; k < 312; ++k) {
            uint64_t y = (g->s[k] & hi) | (g->s[(k + 1) % 312] & lo);
            uint64_t v = g->s[(k + 156) % 312] ^ (y >> 1);
            if (y & 1) v ^= 0xB5026F5AA96619E9ull;
            g->s[k] = v;
        }
        g->i = 0;
    }
    uint64_t x = g->s[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ull;
    x ^= (x << 17) & 0x71D67FFFEDA60000ull;
    x ^= (x << 37) & 0xFFF7EEE000000000ull;
    x ^= x >> 43;
    return x;
}

/* uniform_real_distribution<double>(0,1) over mt19937_64 as libstdc++ (GCC 13) defines it:
 * one engine call, (double)x * 2^-64, clamped below 1. */
static double mt64_uniform(mt64 *g) {
    double u = (double)mt64_next(g) / 18446744073709551616.0;
    if (u >= 1.0) u = nextafter(1.0, 0.0);
    return u;
}

/* Depolarizing error of one trial (5931-5946). */
void jbo_sample(uint64_t base_seed, long long trial_idx, double p, int n, uint8_t *err) {
    static mt64 g; /* not reentrant; the oracle is single-threaded per process */
    mt64_seed(&g, jbo_trial_seed(base_seed, (uint64_t)trial_idx));
    for (int i = 0; i < n; ++i) {
        double u = mt64_uniform(&g);
        if (u < 1.0 - p) {
            err[i] = 0;
        } else {
            double v = (u - (1.0 - p)) / p;
            err[i] = v < 1.0 / 3.0 ? 1 : (v < 2.0 / 3.0 ? 2 : 3);
        }
    }
}

/* ---------------------------------------------------------------- GF(2) row basis */

static int highest_bit(const uint64_t *row, int words) {
    for (int w = words - 1; w >= 0; --w)
        if (row[w]) return w * 64 + 63 - __builtin_clzll(row[w]);
    return -1;
}

/* build_row_basis (845-885). */
int jbo_basis_build(const jbo_code *c, int side, jbo_basis *out) {
    int n = c->n, words = (n + 63) / 64, m = c->m[side];
    memset(out, 0, sizeof(*out));
    out->words = words;
    out->rows = (uint64_t *)calloc((size_t)(m > 0 ? m : 1) * words, sizeof(uint64_t));
    out->pivot = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
    int *p2r = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) p2r[i] = -1;
    uint64_t *row = (uint64_t *)malloc(sizeof(uint64_t) * words);
    for (int ch = 0; ch < m; ++ch) {
        memset(row, 0, sizeof(uint64_t) * words);
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) {
            int v = c->chk_var[side][e];
            row[v >> 6] |= 1ull << (v & 63);
        }
        for (;;) {
            int p = highest_bit(row, words);
            if (p < 0) break;
            if (p2r[p] < 0) {
                memcpy(out->rows + (size_t)out->rank * words, row, sizeof(uint64_t) * words);
                out->pivot[out->rank] = p;
                p2r[p] = out->rank++;
                break;
            }
            const uint64_t *base = out->rows + (size_t)p2r[p] * words;
            for (int w = 0; w < words; ++w) row[w] ^= base[w];
        }
    }
    /* descending pivot order (pivots are distinct) */
    out->order = (int *)malloc(sizeof(int) * (out->rank > 0 ? out->rank : 1));
    int k = 0;
    for (int p = n - 1; p >= 0; --p)
        if (p2r[p] >= 0) out->order[k++] = p2r[p];
    free(p2r);
    free(row);
    return 0;
}

void jbo_basis_free(jbo_basis *b) {
    free(b->rows); free(b->pivot); free(b->order);
    memset(b, 0, sizeof(*b));
}

/* in_row_space (904-920); vec is reduced in place. */
int jbo_in_row_space(const jbo_basis *b, uint64_t *vec) {
    for (int k = 0; k < b->rank; ++k) {
        int r = b->order[k], p = b->pivot[r];
        if (!(vec[p >> 6] & (1ull << (p & 63)))) continue;
        const uint64_t *row = b->rows + (size_t)r * b->words;
        for (int w = 0; w < b->words; ++w) vec[w] ^= row[w];
    }
    for (int w = 0; w < b->words; ++w)
        if (vec[w]) return 0;
    return 1;
}

/* ---------------------------------------------------------------- ETS tables */

static char *trim(char *s) {
    while (*s && isspace((unsigned char)*s)) ++s;
    char *e = s + strlen(s);
    while (e > s && isspace((unsigned char)e[-1])) --e;
    *e = 0;
    return s;
}

/* "V<col>:<idx>" / "C<row>:<idx>" tokens (parse_var_token / parse_check_token, 3181-3197).
 * Tokens whose numbers do not parse are rejected (the reference's std::stoi would throw). */
static int parse_token(const char *tok, char kind, int P, int *id) {
    if (strlen(tok) < 3) return 0;
    if (toupper((unsigned char)tok[0]) != kind) return 0;
    const char *colon = strchr(tok, ':');
    if (!colon) return 0;
    char *end;
    long a = strtol(tok + 1, &end, 10);
    if (end == tok + 1) return 0;
    long b = strtol(colon + 1, &end, 10);
    if (end == colon + 1) return 0;
    *id = (int)(a * P + b);
    return 1;
}

/* split at ',' keeping inner empty tokens, dropping an empty tail (split_csv, 3146-3160). */
static int split_csv(char *s, char **tok, int max) {
    int n = 0;
    char *cur = s;
    for (char *p = s;; ++p) {
        if (*p == ',' || *p == 0) {
            int last = (*p == 0);
            if (!last || p != cur) {
                if (n >= max) return max + 1;
                *p = 0;
                tok[n++] = trim(cur);
            }
            if (last) break;
            cur = p + 1;
        }
    }
    return n;
}

static int cmp_int(const void *a, const void *b) { return (*(const int *)a > *(const int *)b) - (*(const int *)a < *(const int *)b); }

/* read_ets_file (3199-3258). */
int jbo_ets_load(const char *path, int P, int expected_vars, char side, jbo_ets *out) {
    memset(out, 0, sizeof(*out));
    out->var_count = expected_vars;
    if (expected_vars <= 0 || expected_vars > 32) return 1;
    FILE *f = fopen(path, "r");
    if (!f) return 1;
    int cap = 64;
    out->vars = (int *)malloc(sizeof(int) * cap * expected_vars);
    out->key = (uint64_t *)malloc(sizeof(uint64_t) * cap);
    char buf[8192];
    char *tok[64];
    while (fgets(buf, sizeof buf, f)) {
        char *line = trim(buf);
        if (!*line) continue;
        char line_side = 0;
        if (strlen(line) >= 2 && strchr("XxZz", line[0]) && isspace((unsigned char)line[1])) {
            line_side = (char)toupper((unsigned char)line[0]);
            line = trim(line + 1);
        }
        if ((side == 'X' || side == 'Z') && line_side != 0 && line_side != side) continue;
        char *pv = strstr(line, "vars="), *pu = strstr(line, "unsat=");
        if (!pv || !pu || pu < pv + 5) continue;
        *pu = 0;
        char *vars_part = trim(pv + 5);
        char *unsat_part = trim(pu + 6);
        int nv = split_csv(vars_part, tok, 64);
        if (nv != expected_vars) continue;
        int ids[32], ok = 1;
        for (int i = 0; i < nv && ok; ++i) ok = parse_token(tok[i], 'V', P, &ids[i]);
        if (!ok) continue;
        char *ct[4];
        int nc = split_csv(unsat_part, ct, 3);
        if (nc != 2) continue;
        int cks[2];
        if (!parse_token(ct[0], 'C', P, &cks[0]) || !parse_token(ct[1], 'C', P, &cks[1])) continue;
        qsort(ids, nv, sizeof(int), cmp_int);
        if (cks[0] > cks[1]) { int t = cks[0]; cks[0] = cks[1]; cks[1] = t; }
        if (out->count == cap) {
            cap *= 2;
            out->vars = (int *)realloc(out->vars, sizeof(int) * cap * expected_vars);
            out->key = (uint64_t *)realloc(out->key, sizeof(uint64_t) * cap);
        }
        memcpy(out->vars + (size_t)out->count * expected_vars, ids, sizeof(int) * expected_vars);
        out->key[out->count++] = ((uint64_t)(uint32_t)cks[0] << 32) | (uint32_t)cks[1];
    }
    fclose(f);
    return 0;
}

/* ETS groups in the reference order 6, 8, 8p4, 10, 12, ..., 22 (5230-5337, default paths);
 * a group is kept when either side has entries. */
int jbo_ets_set_load_dir(const char *dir, int P, jbo_ets_set *out) {
    memset(out, 0, sizeof(*out));
    static const int sizes[] = {6, 8, 10, 12, 14, 16, 18, 20, 22};
    char path[4096];
    for (int i = 0; i < 9; ++i) {
        for (int pass = 0; pass < (sizes[i] == 8 ? 2 : 1); ++pass) {
            if (pass == 0) snprintf(path, sizeof path, "%s/ets_%d_2.txt", dir, sizes[i]);
            else snprintf(path, sizeof path, "%s/ets_8_2_path4.txt", dir);
            int g = out->ngroups;
            out->size[g] = sizes[i];
            if (pass == 0) snprintf(out->label[g], 8, "%d", sizes[i]);
            else snprintf(out->label[g], 8, "8p4");
            for (int s = 0; s < 2; ++s) {
                jbo_ets *t = &out->tab[g][s];
                if (jbo_ets_load(path, P, sizes[i], s == 0 ? 'X' : 'Z', t) == 0 && t->count > 0) {
                    out->loaded[g][s] = 1;
                } else {
                    free(t->vars); free(t->key);
                    memset(t, 0, sizeof(*t));
                }
            }
            if (out->loaded[g][0] || out->loaded[g][1]) out->ngroups++;
        }
    }
    return 0;
}

int jbo_ets_info(const jbo_ets_set *s, int g, int *size, char *label, int *count_x, int *count_z) {
    if (g >= 0 && g < s->ngroups) {
        if (size) *size = s->size[g];
        if (label) memcpy(label, s->label[g], 8);
        if (count_x) *count_x = s->loaded[g][0] ? s->tab[g][0].count : 0;
        if (count_z) *count_z = s->loaded[g][1] ? s->tab[g][1].count : 0;
    }
    return s->ngroups;
}

void jbo_ets_set_free(jbo_ets_set *s) {
    for (int g = 0; g < s->ngroups; ++g)
        for (int k = 0; k < 2; ++k) { free(s->tab[g][k].vars); free(s->tab[g][k].key); }
    memset(s, 0, sizeof(*s));
}

/* Gauss-Jordan over <=32 columns (solve_gf2, 3357-3391); free variables set to 0. */
static int solve_gf2_32(uint32_t *a, int *b, int m, int nvars, int *sol) {
    int where[32];
    for (int c = 0; c < nvars; ++c) where[c] = -1;
    int r = 0;
    for (int c = 0; c < nvars && r < m; ++c) {
        int sel = r;
        while (sel < m && !((a[sel] >> c) & 1u)) ++sel;
        if (sel == m) continue;
        uint32_t ta = a[sel]; a[sel] = a[r]; a[r] = ta;
        int tb = b[sel]; b[sel] = b[r]; b[r] = tb;
        where[c] = r;
        for (int i = 0; i < m; ++i)
            if (i != r && ((a[i] >> c) & 1u)) { a[i] ^= a[r]; b[i] ^= b[r]; }
        ++r;
    }
    for (int i = r; i < m; ++i)
        if (a[i] == 0 && b[i]) return 0;
    for (int c = 0; c < nvars; ++c) sol[c] = where[c] >= 0 ? (b[where[c]] & 1) : 0;
    return 1;
}

static uint8_t flip_state(int side, uint8_t s) { return (uint8_t)(side == 0 ? (s ^ 1) : (s ^ 2)); }

/* attempt_ets_fix_side (3525-3642). */
static int ets_fix_side(const jbo_code *c, const jbo_ets *t, int side, const uint8_t *target, uint8_t *est,
                        uint8_t *diff, uint8_t *trial) {
    if (t->count == 0) return 0;
    int nv = t->var_count;
    if (nv <= 0 || nv > 32) return 0;
    int nus = 0, us[2] = {0, 0};
    for (int ch = 0; ch < c->m[side]; ++ch) {
        int par = 0;
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) par ^= sbit(side, est[c->chk_var[side][e]]);
        diff[ch] = (uint8_t)(par ^ target[ch]);
        if (diff[ch]) { if (nus < 2) us[nus] = ch; nus++; }
    }
    if (nus != 2) return 0;
    int c0 = us[0] < us[1] ? us[0] : us[1], c1 = us[0] < us[1] ? us[1] : us[0];
    uint64_t key = ((uint64_t)(uint32_t)c0 << 32) | (uint32_t)c1;
    int checks[32 * 16];
    uint32_t rows[32 * 16];
    int rhs[32 * 16], delta[32];
    for (int k = 0; k < t->count; ++k) {
        if (t->key[k] != key) continue;
        const int *vars = t->vars + (size_t)k * nv;
        int nch = 0;
        for (int i = 0; i < nv; ++i) {
            int v = vars[i];
            for (int q = c->var_off[side][v]; q < c->var_off[side][v + 1]; ++q) {
                int e = c->var_edge[side][q], ch = 0;
                /* check of edge e: binary search in chk_off */
                int lo = 0, hi = c->m[side] - 1;
                while (lo < hi) { int mid = (lo + hi + 1) / 2; if (c->chk_off[side][mid] <= e) lo = mid; else hi = mid - 1; }
                ch = lo;
                int seen = 0;
                for (int j = 0; j < nch; ++j) if (checks[j] == ch) { seen = 1; break; }
                if (!seen && nch < 32 * 16) checks[nch++] = ch;
            }
        }
        int ok = 1;
        for (int j = 0; j < nch && ok; ++j)
            if (diff[checks[j]] && checks[j] != c0 && checks[j] != c1) ok = 0;
        if (!ok) continue;
        int nr = 0;
        for (int j = 0; j < nch; ++j) {
            uint32_t mask = 0;
            int ch = checks[j];
            for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) {
                int v = c->chk_var[side][e];
                for (int i = 0; i < nv; ++i) if (vars[i] == v) { mask |= 1u << i; break; }
            }
            if (!mask) continue;
            rows[nr] = mask;
            rhs[nr++] = diff[ch] & 1;
        }
        if (!solve_gf2_32(rows, rhs, nr, nv, delta)) continue;
        memcpy(trial, est, (size_t)c->n);
        for (int i = 0; i < nv; ++i) if (delta[i]) trial[vars[i]] = flip_state(side, trial[vars[i]]);
        if (syn_equal(c, side, trial, target)) {
            memcpy(est, trial, (size_t)c->n);
            return 1;
        }
    }
    return 0;
}

/* attempt_ets_fix_side_multi (3644-3668): first group that applies wins. */
int jbo_ets_fix_multi(const jbo_code *c, const jbo_ets_set *ets, int side, const uint8_t *target, uint8_t *est,
                      int *applied_size, int *applied_group) {
    *applied_size = 0;
    *applied_group = -1;
    if (!ets) return 0;
    uint8_t *diff = (uint8_t *)malloc(c->m[side]);
    uint8_t *trial = (uint8_t *)malloc(c->n);
    int applied = 0;
    for (int g = 0; g < ets->ngroups; ++g) {
        if (!ets->loaded[g][side]) continue;
        if (ets_fix_side(c, &ets->tab[g][side], side, target, est, diff, trial)) {
            applied = 1;
            *applied_size = ets->size[g];
            *applied_group = g;
            break;
        }
    }
    free(diff);
    free(trial);
    return applied;
}

/* ---------------------------------------------------------------- GF(2) on bit rows */

typedef struct { int solvable, rank, unique; } gf2_info;

/* solve_gf2_bits (3408-3462): Gauss-Jordan, first pivot row at or below r; sol gets the
 * solution with free variables 0.  If where_out is given it receives the pivot row of
 * each column (or -1) and rows/rhs are left reduced. */
static gf2_info solve_gf2_bits(uint64_t *rows, int *rhs, int m, int nvars, int *sol, int *where_out) {
    gf2_info info = {0, 0, 0};
    if (nvars <= 0) return info;
    int words = (nvars + 63) / 64;
    int *where = where_out ? where_out : (int *)malloc(sizeof(int) * nvars);
    for (int c = 0; c < nvars; ++c) where[c] = -1;
    int r = 0;
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * words);
    for (int c = 0; c < nvars && r < m; ++c) {
        int w = c >> 6;
        uint64_t mask = 1ull << (c & 63);
        int sel = r;
        while (sel < m && !(rows[(size_t)sel * words + w] & mask)) ++sel;
        if (sel == m) continue;
        if (sel != r) {
            memcpy(tmp, rows + (size_t)sel * words, sizeof(uint64_t) * words);
            memcpy(rows + (size_t)sel * words, rows + (size_t)r * words, sizeof(uint64_t) * words);
            memcpy(rows + (size_t)r * words, tmp, sizeof(uint64_t) * words);
            int t = rhs[sel]; rhs[sel] = rhs[r]; rhs[r] = t;
        }
        where[c] = r;
        const uint64_t *pr = rows + (size_t)r * words;
        for (int i = 0; i < m; ++i) {
            if (i == r) continue;
            uint64_t *ri = rows + (size_t)i * words;
            if (!(ri[w] & mask)) continue;
            for (int k = w; k < words; ++k) ri[k] ^= pr[k]; /* columns < c of the pivot row are 0 */
            rhs[i] ^= rhs[r];
        }
        ++r;
    }
    free(tmp);
    int bad = 0;
    for (int i = r; i < m && !bad; ++i) {
        int zero = 1;
        for (int k = 0; k < words; ++k) if (rows[(size_t)i * words + k]) { zero = 0; break; }
        if (zero && (rhs[i] & 1)) bad = 1;
    }
    info.rank = r;
    if (!bad) {
        info.solvable = 1;
        info.unique = (r == nvars);
        if (sol) for (int c = 0; c < nvars; ++c) sol[c] = where[c] >= 0 ? (rhs[where[c]] & 1) : 0;
    }
    if (!where_out) free(where);
    return info;
}

static int build_sub_rows(const jbo_code *c, int side, const int *pos, int ncols, const uint8_t *diff, uint64_t *rows,
                          int *rhs, int *nrows) {
    int words = (ncols + 63) / 64, nr = 0;
    for (int ch = 0; ch < c->m[side]; ++ch) {
        uint64_t *row = rows + (size_t)nr * words;
        memset(row, 0, sizeof(uint64_t) * words);
        int any = 0;
        for (int e = c->chk_off[side][ch]; e < c->chk_off[side][ch + 1]; ++e) {
            int p = pos[c->chk_var[side][e]];
            if (p < 0) continue;
            row[p >> 6] |= 1ull << (p & 63);
            any = 1;
        }
        if (!any) {
            if (diff[ch]) { *nrows = nr; return 0; }
            continue;
        }
        rhs[nr++] = diff[ch] & 1;
    }
    *nrows = nr;
    return 1;
}

/* attempt_flip_pp_side (3726-3880) without its logging; applies only a unique solution
 * that reproduces the target syndrome. */
int jbo_flip_pp(const jbo_code *c, int side, const int *vars_in, int nv_in, const uint8_t *target, uint8_t *est) {
    if (nv_in <= 0) return 0;
    int n = c->n;
    int *vars = (int *)malloc(sizeof(int) * nv_in);
    int nv = 0;
    for (int i = 0; i < nv_in; ++i) if (vars_in[i] >= 0 && vars_in[i] < n) vars[nv++] = vars_in[i];
    if (nv == 0) { free(vars); return 0; }
    qsort(vars, nv, sizeof(int), cmp_int);
    int u = 0;
    for (int i = 0; i < nv; ++i) if (i == 0 || vars[i] != vars[i - 1]) vars[u++] = vars[i];
    nv = u;
    int m = c->m[side];
    uint8_t *diff = (uint8_t *)malloc(m);
    jbo_syndrome(c, side, est, diff);
    for (int ch = 0; ch < m; ++ch) diff[ch] ^= target[ch];
    int *pos = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) pos[i] = -1;
    for (int i = 0; i < nv; ++i) pos[vars[i]] = i;
    int words = (nv + 63) / 64;
    uint64_t *rows = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(m > 0 ? m : 1) * words);
    int *rhs = (int *)malloc(sizeof(int) * (m > 0 ? m : 1));
    int *delta = (int *)malloc(sizeof(int) * nv);
    int nr = 0, applied = 0;
    if (build_sub_rows(c, side, pos, nv, diff, rows, rhs, &nr) && nr > 0) {
        gf2_info info = solve_gf2_bits(rows, rhs, nr, nv, delta, NULL);
        if (info.solvable && info.unique) {
            uint8_t *trial = (uint8_t *)malloc(n);
            memcpy(trial, est, n);
            for (int i = 0; i < nv; ++i) if (delta[i]) trial[vars[i]] = flip_state(side, trial[vars[i]]);
            if (syn_equal(c, side, trial, target)) { memcpy(est, trial, n); applied = 1; }
            free(trial);
        }
    }
    free(vars); free(diff); free(pos); free(rows); free(rhs); free(delta);
    return applied;
}

/* ---------------------------------------------------------------- OSD */

typedef struct { int computed, solvable, rank, unique; } osd_info;

/* solve_osd_pp_for_k (3882-3949) reduced to its outcome; delta (k entries) when wanted. */
static osd_info osd_solve_k(const jbo_code *c, int side, const int *order, int k, const uint8_t *diff, int *pos,
                            uint64_t *rows, int *rhs, int *delta) {
    osd_info info = {1, 0, 0, 0};
    int n = c->n;
    if (k <= 0 || n < k) return info;
    for (int i = 0; i < n; ++i) pos[i] = -1;
    for (int i = 0; i < k; ++i) pos[order[i]] = i;
    int nr = 0;
    if (!build_sub_rows(c, side, pos, k, diff, rows, rhs, &nr)) return info;
    if (nr == 0) {
        info.solvable = 1;
        info.unique = (k == 0);
        if (delta) for (int i = 0; i < k; ++i) delta[i] = 0;
        return info;
    }
    gf2_info g = solve_gf2_bits(rows, rhs, nr, k, delta, NULL);
    info.solvable = g.solvable;
    info.rank = g.rank;
    info.unique = g.unique;
    return info;
}

static const double *g_sort_llr;
static int cmp_llr(const void *pa, const void *pb) {
    int a = *(const int *)pa, b = *(const int *)pb;
    double x = g_sort_llr[a], y = g_sort_llr[b];
    if (x == y) return (a > b) - (a < b);
    return x < y ? -1 : 1;
}

/* attempt_osd_pp_side (4078-4386).  The min-dof fallback after the unique-K search is
 * unreachable in the reference (k_use is always a K whose system was unique), so the
 * outcome is decided by the two binary searches and the weight-30 rule. */
int jbo_osd_pp(const jbo_code *c, int side, const double *abs_llr, const uint8_t *target, uint8_t *est) {
    int n = c->n, m = c->m[side];
    if (!abs_llr || m == 0 || n <= 0) return 0;
    uint8_t *diff = (uint8_t *)malloc(m);
    jbo_syndrome(c, side, est, diff);
    int any = 0;
    for (int ch = 0; ch < m; ++ch) { diff[ch] ^= target[ch]; any |= diff[ch]; }
    if (!any) { free(diff); return 0; }
    int *order = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) order[i] = i;
    g_sort_llr = abs_llr;
    qsort(order, n, sizeof(int), cmp_llr); /* total order (index tie-break) = stable_sort result */
    int words = (n + 63) / 64;
    uint64_t *rows = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)m * words);
    int *rhs = (int *)malloc(sizeof(int) * m);
    int *pos = (int *)malloc(sizeof(int) * n);
    osd_info *cache = (osd_info *)calloc((size_t)n + 1, sizeof(osd_info));
#define OSD_GET(K) (cache[K].computed ? cache[K] : (cache[K] = osd_solve_k(c, side, order, (K), diff, pos, rows, rhs, NULL)))
    int applied = 0;
    int k_max = n;
    if (OSD_GET(k_max).solvable) {
        int lo = 1, hi = k_max;
        while (lo < hi) {
            int mid = lo + (hi - lo) / 2;
            if (OSD_GET(mid).solvable) hi = mid; else lo = mid + 1;
        }
        int k_solve = lo;
        if (OSD_GET(k_solve).unique) {
            int lo2 = k_solve, hi2 = k_max;
            while (lo2 < hi2) {
                int mid = lo2 + (hi2 - lo2 + 1) / 2;
                if (OSD_GET(mid).unique) lo2 = mid; else hi2 = mid - 1;
            }
            int k_use = lo2;
            int *delta = (int *)malloc(sizeof(int) * k_use);
            osd_info iu = osd_solve_k(c, side, order, k_use, diff, pos, rows, rhs, delta);
            if (iu.solvable && iu.unique) {
                uint8_t *trial = (uint8_t *)malloc(n);
                memcpy(trial, est, n);
                int weight = 0;
                for (int i = 0; i < k_use; ++i) if (delta[i] & 1) { weight++; trial[order[i]] = flip_state(side, trial[order[i]]); }
                if (syn_equal(c, side, trial, target) && weight <= 30) { memcpy(est, trial, n); applied = 1; }
                free(trial);
            }
            free(delta);
        }
    }
#undef OSD_GET
    free(diff); free(order); free(rows); free(rhs); free(pos); free(cache);
    return applied;
}

/* ---------------------------------------------------------------- joint BP */

struct jbo_work {
    int n, e[2];
    double *v2c[2], *c2v[2];       /* 4 doubles per edge */
    uint8_t *est, *prev, *pprev, *trial;
    double *llr[2];
    /* flip window: ring of per-iteration flag arrays per side */
    int win_cap, win_len[2], win_head[2];
    uint8_t *win[2];
    uint8_t *last_flip[2];          /* flags of the last iteration's flips */
    int have_last;
    int flip_active;               /* window recorded (stagnation seen and flip_hist > 0) */
    int *us_hist, us_len, us_head;
    uint8_t *shx, *shz;
    int *setbuf;
};

jbo_work *jbo_work_new(const jbo_code *c) {
    jbo_work *w = (jbo_work *)calloc(1, sizeof(jbo_work));
    w->n = c->n;
    for (int s = 0; s < 2; ++s) {
        w->e[s] = c->e[s];
        w->v2c[s] = (double *)malloc(sizeof(double) * 4 * (c->e[s] > 0 ? c->e[s] : 1));
        w->c2v[s] = (double *)malloc(sizeof(double) * 4 * (c->e[s] > 0 ? c->e[s] : 1));
        w->llr[s] = (double *)malloc(sizeof(double) * c->n);
        w->last_flip[s] = (uint8_t *)malloc(c->n);
    }
    w->est = (uint8_t *)malloc(c->n);
    w->prev = (uint8_t *)malloc(c->n);
    w->pprev = (uint8_t *)malloc(c->n);
    w->trial = (uint8_t *)malloc(c->n);
    w->us_hist = (int *)malloc(sizeof(int) * 100);
    w->shx = (uint8_t *)malloc(c->m[0] > 0 ? c->m[0] : 1);
    w->shz = (uint8_t *)malloc(c->m[1] > 0 ? c->m[1] : 1);
    w->setbuf = (int *)malloc(sizeof(int) * c->n);
    return w;
}

void jbo_work_free(jbo_work *w) {
    if (!w) return;
    for (int s = 0; s < 2; ++s) { free(w->v2c[s]); free(w->c2v[s]); free(w->llr[s]); free(w->win[s]); free(w->last_flip[s]); }
    free(w->est); free(w->prev); free(w->pprev); free(w->trial); free(w->us_hist); free(w->shx); free(w->shz);
    free(w->setbuf);
    free(w);
}

/* normalize_msg (650-657): divide by ((m0+m1)+m2)+m3, uniform when the sum is <= 0. */
static void norm4(double *m) {
    double s = m[0] + m[1];
    s = s + m[2];
    s = s + m[3];
    if (s <= 0.0) { m[0] = m[1] = m[2] = m[3] = 0.25; return; }
    m[0] = m[0] / s; m[1] = m[1] / s; m[2] = m[2] / s; m[3] = m[3] / s;
}

/* Check-node update of one side (X: 2373-2410, Z: 2412-2449): parity product of the
 * binary marginals with prefix/suffix passes, output {v0,v1,v0,v1} (X) or {v0,v0,v1,v1} (Z). */
static void check_update(const jbo_code *c, int side, const uint8_t *syn, const double *v2c, double *c2v) {
    double q0[64], q1[64], pe[65], po[65], se[65], so[65];
    for (int ch = 0; ch < c->m[side]; ++ch) {
        int b = c->chk_off[side][ch], deg = c->chk_off[side][ch + 1] - b;
        for (int i = 0; i < deg; ++i) {
            const double *m = v2c + 4 * (size_t)(b + i);
            if (side == 0) { q0[i] = m[0] + m[2]; q1[i] = m[1] + m[3]; }
            else { q0[i] = m[0] + m[1]; q1[i] = m[2] + m[3]; }
        }
        pe[0] = 1.0; po[0] = 0.0;
        for (int i = 0; i < deg; ++i) {
            double ne = pe[i] * q0[i] + po[i] * q1[i];
            double no = pe[i] * q1[i] + po[i] * q0[i];
            pe[i + 1] = ne; po[i + 1] = no;
        }
        se[deg] = 1.0; so[deg] = 0.0;
        for (int i = deg - 1; i >= 0; --i) {
            double ne = se[i + 1] * q0[i] + so[i + 1] * q1[i];
            double no = se[i + 1] * q1[i] + so[i + 1] * q0[i];
            se[i] = ne; so[i] = no;
        }
        for (int i = 0; i < deg; ++i) {
            double p_even = pe[i] * se[i + 1] + po[i] * so[i + 1];
            double p_odd = pe[i] * so[i + 1] + po[i] * se[i + 1];
            double v0 = syn[ch] == 0 ? p_even : p_odd;
            double v1 = syn[ch] == 0 ? p_odd : p_even;
            double *o = c2v + 4 * (size_t)(b + i);
            if (side == 0) { o[0] = v0; o[1] = v1; o[2] = v0; o[3] = v1; }
            else { o[0] = v0; o[1] = v0; o[2] = v1; o[3] = v1; }
            norm4(o);
        }
    }
}

static void mul4(const double *a, const double *b, double *o) {
    o[0] = a[0] * b[0]; o[1] = a[1] * b[1]; o[2] = a[2] * b[2]; o[3] = a[3] * b[3];
}

/* scaled_mix (1903-1911). */
static void damp_store(double *dst, const double *nw, double d) {
    if (d <= 0.0) { memcpy(dst, nw, 4 * sizeof(double)); return; }
    double o[4];
    for (int i = 0; i < 4; ++i) o[i] = (1.0 - d) * nw[i] + d * dst[i];
    norm4(o);
    memcpy(dst, o, sizeof o);
}

/* Variable-node update (2451-2519): prefix/suffix products over the X and Z edges,
 * total = normalize(prior * (PX * PZ)), est = first argmax, |LLR| when requested,
 * extrinsic v2c = normalize((prior * excl) * other-side total) with damping. */
static void var_update(const jbo_code *c, const double *prior, jbo_work *w, int upd_x, int upd_z, int collect_llr,
                       double damping) {
    double px[17][4], sx_[17][4], pz[17][4], sz_[17][4];
    for (int v = 0; v < c->n; ++v) {
        int bx = c->var_off[0][v], dx = c->var_off[0][v + 1] - bx;
        int bz = c->var_off[1][v], dz = c->var_off[1][v + 1] - bz;
        for (int j = 0; j < 4; ++j) px[0][j] = sx_[dx][j] = pz[0][j] = sz_[dz][j] = 1.0;
        for (int i = 0; i < dx; ++i) mul4(px[i], w->c2v[0] + 4 * (size_t)c->var_edge[0][bx + i], px[i + 1]);
        for (int i = dx - 1; i >= 0; --i) mul4(sx_[i + 1], w->c2v[0] + 4 * (size_t)c->var_edge[0][bx + i], sx_[i]);
        for (int i = 0; i < dz; ++i) mul4(pz[i], w->c2v[1] + 4 * (size_t)c->var_edge[1][bz + i], pz[i + 1]);
        for (int i = dz - 1; i >= 0; --i) mul4(sz_[i + 1], w->c2v[1] + 4 * (size_t)c->var_edge[1][bz + i], sz_[i]);
        double xz[4], tot[4];
        mul4(px[dx], pz[dz], xz);
        mul4(prior, xz, tot);
        norm4(tot);
        int best = 0;
        for (int s = 1; s < 4; ++s) if (tot[s] > tot[best]) best = s;
        w->est[v] = (uint8_t)best;
        if (collect_llr) {
            const double eps = 1e-300;
            double px1 = tot[1] + tot[3], px0 = tot[0] + tot[2];
            double pz1 = tot[2] + tot[3], pz0 = tot[0] + tot[1];
            double lx = log(px1 > eps ? px1 : eps) - log(px0 > eps ? px0 : eps);
            double lz = log(pz1 > eps ? pz1 : eps) - log(pz0 > eps ? pz0 : eps);
            w->llr[0][v] = fabs(lx);
            w->llr[1][v] = fabs(lz);
        }
        if (upd_x) {
            for (int i = 0; i < dx; ++i) {
                double ex[4], o[4], o2[4];
                mul4(px[i], sx_[i + 1], ex);
                mul4(prior, ex, o);
                mul4(o, pz[dz], o2);
                norm4(o2);
                damp_store(w->v2c[0] + 4 * (size_t)c->var_edge[0][bx + i], o2, damping);
            }
        }
        if (upd_z) {
            for (int i = 0; i < dz; ++i) {
                double ez[4], o[4], o2[4];
                mul4(pz[i], sz_[i + 1], ez);
                mul4(prior, px[dx], o);
                mul4(o, ez, o2);
                norm4(o2);
                damp_store(w->v2c[1] + 4 * (size_t)c->var_edge[1][bz + i], o2, damping);
            }
        }
    }
}

/* freeze_side_msgs with det_msg_xbit/zbit (1876-1901). */
static void freeze_side(const jbo_code *c, int side, jbo_work *w) {
    for (int e = 0; e < c->e[side]; ++e) {
        int bit = sbit(side, w->est[c->chk_var[side][e]]);
        double m[4];
        if (side == 0) { m[0] = bit ? 0.0 : 0.5; m[1] = bit ? 0.5 : 0.0; m[2] = m[0]; m[3] = m[1]; }
        else { m[0] = bit ? 0.0 : 0.5; m[1] = m[0]; m[2] = bit ? 0.5 : 0.0; m[3] = m[2]; }
        memcpy(w->v2c[side] + 4 * (size_t)e, m, sizeof m);
        memcpy(w->c2v[side] + 4 * (size_t)e, m, sizeof m);
    }
}

/* detect_us_oscillation (2021-2053): full 100-sample window, range >= max(10, 0.2*mean),
 * at least two direction changes. */
static int us_oscillation(const jbo_work *w) {
    if (w->us_len < 100) return 0;
    int first = w->us_hist[w->us_head % 100];
    int mn = first, mx = first;
    long long sum = 0;
    for (int k = 0; k < 100; ++k) {
        int v = w->us_hist[(w->us_head + k) % 100];
        if (v < mn) mn = v;
        if (v > mx) mx = v;
        sum += v;
    }
    double mean = (double)sum / 100.0;
    int range = mx - mn;
    if (mean <= 0.0) return 0;
    int min_range = (int)(mean * 0.2);
    if (min_range < 10) min_range = 10;
    if (range < min_range) return 0;
    int prev_sign = 0, turns = 0;
    for (int k = 1; k < 100; ++k) {
        int d = w->us_hist[(w->us_head + k) % 100] - w->us_hist[(w->us_head + k - 1) % 100];
        int sg = d > 0 ? 1 : (d < 0 ? -1 : 0);
        if (sg) {
            if (prev_sign && sg != prev_sign) turns++;
            prev_sign = sg;
        }
    }
    return turns >= 2;
}

static int list_from_flags(const uint8_t *f, int n, int *out) {
    int k = 0;
    for (int i = 0; i < n; ++i) if (f[i]) out[k++] = i;
    return k;
}

/* One side's flip-PP candidate sets (build_flip_sets, 3670-3689), tried in order until one
 * applies. window entries are oldest->newest; sets: union, then newest->oldest non-empty
 * entries; "last" only when there is no window and no union. */
static int flip_side(const jbo_code *c, jbo_work *w, int side, int hist_active, const uint8_t *target, uint8_t *est) {
    int n = c->n, *buf = w->setbuf, applied = 0;
    int have_window = hist_active && w->win_cap > 0;
    int nunion = 0;
    if (have_window) {
        uint8_t *u = (uint8_t *)calloc(n, 1);
        for (int k = 0; k < w->win_len[side]; ++k) {
            const uint8_t *f = w->win[side] + (size_t)((w->win_head[side] + k) % w->win_cap) * n;
            for (int i = 0; i < n; ++i) u[i] |= f[i];
        }
        nunion = list_from_flags(u, n, buf);
        free(u);
        if (nunion > 0 && jbo_flip_pp(c, side, buf, nunion, target, est)) return 1;
    }
    int wlen = have_window ? w->win_len[side] : 0;
    if (wlen > 0) {
        for (int k = wlen - 1; k >= 0 && !applied; --k) {
            const uint8_t *f = w->win[side] + (size_t)((w->win_head[side] + k) % w->win_cap) * n;
            int cnt = list_from_flags(f, n, buf);
            if (cnt > 0 && jbo_flip_pp(c, side, buf, cnt, target, est)) applied = 1;
        }
    } else if (nunion == 0 && w->have_last) {
        int cnt = list_from_flags(w->last_flip[side], n, buf);
        if (cnt > 0 && jbo_flip_pp(c, side, buf, cnt, target, est)) applied = 1;
    }
    return applied;
}

/* joint_bp_decode (1943-3079) without its logging. */
int jbo_decode(const jbo_code *c, const jbo_ets_set *ets, jbo_work *w, const uint8_t *sx, const uint8_t *sz,
               double p, int max_iter, int flip_hist, int freeze_syn, double damping, int enable_pp,
               uint8_t *est_out, double *abs_llr_x, double *abs_llr_z, jbo_result *res) {
    int n = c->n;
    memset(res, 0, sizeof(*res));
    double prior[4] = {1.0 - p, p / 3.0, p / 3.0, p / 3.0};
    norm4(prior);
    for (int s = 0; s < 2; ++s)
        for (int e = 0; e < c->e[s]; ++e) {
            memcpy(w->v2c[s] + 4 * (size_t)e, prior, sizeof prior);
            for (int j = 0; j < 4; ++j) w->c2v[s][4 * (size_t)e + j] = 0.25;
        }
    memset(w->est, 0, n);
    int hist_window = flip_hist > 0 ? flip_hist : 0;
    if (w->win_cap != hist_window) {
        for (int s = 0; s < 2; ++s) {
            free(w->win[s]);
            w->win[s] = hist_window ? (uint8_t *)malloc((size_t)hist_window * n) : NULL;
        }
        w->win_cap = hist_window;
    }
    w->win_len[0] = w->win_len[1] = w->win_head[0] = w->win_head[1] = 0;
    w->have_last = 0;
    w->us_len = w->us_head = 0;
    int have_prev = 0, have_pprev = 0;
    int flip_active = 0, freeze_x = 0, freeze_z = 0;
    int stall_same = 0, stall_active = 0, osc_active = 0, usosc_active = 0;
    int llr_valid = 0, iters = max_iter, done = 0;

    for (int iter = 0; iter < max_iter && !done; ++iter) {
        int collect_llr = enable_pp || ((abs_llr_x != NULL) && iter + 1 == max_iter);
        if (!freeze_x) check_update(c, 0, sx, w->v2c[0], w->c2v[0]);
        if (!freeze_z) check_update(c, 1, sz, w->v2c[1], w->c2v[1]);
        var_update(c, prior, w, !freeze_x, !freeze_z, collect_llr, damping);
        if (collect_llr) llr_valid = 1;
        jbo_syndrome(c, 0, w->est, w->shx);
        jbo_syndrome(c, 1, w->est, w->shz);
        int syn_x = memcmp(w->shx, sx, c->m[0]) == 0, syn_z = memcmp(w->shz, sz, c->m[1]) == 0;
        int syn_all = syn_x && syn_z;
        if (freeze_syn) {
            if (syn_x && !freeze_x) { freeze_x = 1; freeze_side(c, 0, w); }
            if (syn_z && !freeze_z) { freeze_z = 1; freeze_side(c, 1, w); }
        }
        int pp_skip = 0;
        if (!syn_all) {
            int ux = 0, uz = 0;
            for (int i = 0; i < c->m[0]; ++i) ux += w->shx[i] != sx[i];
            for (int i = 0; i < c->m[1]; ++i) uz += w->shz[i] != sz[i];
            int sig = ux > uz ? ux : uz;
            pp_skip = sig > 20;
            if (w->us_len < 100) w->us_hist[(w->us_head + w->us_len++) % 100] = sig;
            else { w->us_hist[w->us_head] = sig; w->us_head = (w->us_head + 1) % 100; }
        }
        int same_est = have_prev && memcmp(w->est, w->prev, n) == 0;
        int oscillating = have_pprev && memcmp(w->est, w->pprev, n) == 0 && !same_est;
        if (!syn_all) {
            int allow = (iter + 1 >= 100) || (iter + 1 == max_iter);
            stall_same = same_est ? stall_same + 1 : 0;
            int activate = 0;
            if (!stall_active && (stall_same >= 1 || iter + 1 == max_iter) && allow) { stall_active = 1; activate = 1; }
            if (!osc_active && oscillating && allow) { osc_active = 1; activate = 1; }
            if (!usosc_active && allow && us_oscillation(w)) { usosc_active = 1; activate = 1; }
            if (activate && !flip_active && hist_window > 0) {
                flip_active = 1;
                w->win_len[0] = w->win_len[1] = w->win_head[0] = w->win_head[1] = 0;
            }
        }
        if (have_prev) {
            for (int s = 0; s < 2; ++s)
                for (int i = 0; i < n; ++i) w->last_flip[s][i] = (uint8_t)(sbit(s, w->prev[i]) != sbit(s, w->est[i]));
            w->have_last = 1;
            if (flip_active) {
                for (int s = 0; s < 2; ++s) {
                    int slot;
                    if (w->win_len[s] < hist_window) slot = (w->win_head[s] + w->win_len[s]++) % hist_window;
                    else { slot = w->win_head[s]; w->win_head[s] = (w->win_head[s] + 1) % hist_window; }
                    memcpy(w->win[s] + (size_t)slot * n, w->last_flip[s], n);
                }
            }
        }
        if (syn_all) {
            iters = iter + 1;
            res->bp_ok = 1;
            res->syndrome_ok = 1;
            done = 1;
            break;
        }
        if (enable_pp && (stall_active || osc_active || usosc_active) && !pp_skip) {
            uint8_t *tr = w->trial;
            memcpy(tr, w->est, n);
            int ok = 0, ets_ok = 0, flip_ok = 0;
            int sx_size, sx_grp, sz_size, sz_grp;
            int fx = jbo_ets_fix_multi(c, ets, 0, sx, tr, &sx_size, &sx_grp);
            int fz = jbo_ets_fix_multi(c, ets, 1, sz, tr, &sz_size, &sz_grp);
            int ets_used = fx || fz;
            int ets6 = sx_size == 6 || sz_size == 6, ets12 = sx_size == 12 || sz_size == 12;
            unsigned mask = 0;
            if (fx) mask |= 1u << sx_grp;
            if (fz) mask |= 1u << sz_grp;
            if (ets_used) {
                ok = syn_equal(c, 0, tr, sx) && syn_equal(c, 1, tr, sz);
                if (ok) ets_ok = 1;
            }
            if (!ok) {
                int ax = flip_side(c, w, 0, flip_active, sx, tr);
                int az = flip_side(c, w, 1, flip_active, sz, tr);
                if (ax || az) {
                    ok = syn_equal(c, 0, tr, sx) && syn_equal(c, 1, tr, sz);
                    if (ok) flip_ok = 1;
                }
            }
            if (!ok) {
                int ux = unsat_count(c, 0, tr, sx), uz = unsat_count(c, 1, tr, sz);
                if ((ux > uz ? ux : uz) <= 20) {
                    int ox = jbo_osd_pp(c, 0, w->llr[0], sx, tr);
                    int oz = jbo_osd_pp(c, 1, w->llr[1], sz, tr);
                    if (ox || oz) ok = syn_equal(c, 0, tr, sx) && syn_equal(c, 1, tr, sz);
                }
            }
            if (ok) {
                memcpy(w->est, tr, n);
                iters = iter + 1;
                res->syndrome_ok = 1;
                res->pp_success = 1;
                res->pp_success_ets = ets_ok;
                res->pp_success_flip = flip_ok;
                res->pp_used_ets_any = ets_used;
                res->pp_used_ets6 = ets6;
                res->pp_used_ets12 = ets12;
                res->ets_label_mask = ets_used ? mask : 0;
                done = 1;
                break;
            }
        }
        memcpy(w->pprev, w->prev, n);
        have_pprev = have_prev;
        memcpy(w->prev, w->est, n);
        have_prev = 1;
    }
    res->iterations = iters;
    memcpy(est_out, w->est, n);
    if (abs_llr_x && llr_valid) {
        memcpy(abs_llr_x, w->llr[0], sizeof(double) * n);
        memcpy(abs_llr_z, w->llr[1], sizeof(double) * n);
    }
    /* flip data for post-BP PP stays in w: window (valid when active) and last flips */
    w->flip_active = flip_active;
    return 0;
}

/* ---------------------------------------------------------------- Monte-Carlo trial */

/* One trial of the simulate loop body (5947-6245) from a known error. */
int jbo_error_trial(const jbo_code *c, const jbo_ets_set *ets, const jbo_basis *bx, const jbo_basis *bz,
                    jbo_work *w, const uint8_t *err_in, long long trial_idx, double p, int max_iter, int flip_hist,
                    double damping, int freeze_syn, int enable_pp, jbo_trial_record *rec, uint8_t *est_out) {
    int n = c->n;
    uint8_t *err = (uint8_t *)malloc(n), *est = (uint8_t *)malloc(n);
    uint8_t *sx = (uint8_t *)malloc(c->m[0]), *sz = (uint8_t *)malloc(c->m[1]);
    double *lx = (double *)malloc(sizeof(double) * n), *lz = (double *)malloc(sizeof(double) * n);
    memcpy(err, err_in, n);
    jbo_syndrome(c, 0, err, sx);
    jbo_syndrome(c, 1, err, sz);
    jbo_result r;
    jbo_decode(c, ets, w, sx, sz, p, max_iter, flip_hist, freeze_syn, damping, enable_pp, est,
               enable_pp ? lx : NULL, enable_pp ? lz : NULL, &r);
    int used6 = r.pp_used_ets6, used12 = r.pp_used_ets12;
    int used_any = r.pp_used_ets_any || used6 || used12;
    int ok = r.syndrome_ok, ets_ok = r.pp_success_ets, flip_ok = r.pp_success_flip, osd_ok = 0, ets_applied = 0;
    /* post-BP stages (6020-6197) */
    if (!ok && enable_pp) {
        int szx, gx, szz, gz;
        int fx = jbo_ets_fix_multi(c, ets, 0, sx, est, &szx, &gx);
        int fz = jbo_ets_fix_multi(c, ets, 1, sz, est, &szz, &gz);
        ets_applied = fx || fz;
        used_any = used_any || ets_applied;
        used6 = used6 || szx == 6 || szz == 6;
        used12 = used12 || szx == 12 || szz == 12;
        if (ets_applied) {
            ok = syn_equal(c, 0, est, sx) && syn_equal(c, 1, est, sz);
            if (ok) ets_ok = 1;
        }
    }
    if (!ok && enable_pp) {
        /* the decode left the flip window (if active) and the last flips in w */
        int ax = flip_side(c, w, 0, w->flip_active, sx, est);
        int az = flip_side(c, w, 1, w->flip_active, sz, est);
        if (ax || az) {
            ok = syn_equal(c, 0, est, sx) && syn_equal(c, 1, est, sz);
            if (ok) flip_ok = 1;
        }
    }
    if (!ok && enable_pp) {
        int ux = unsat_count(c, 0, est, sx), uz = unsat_count(c, 1, est, sz);
        if ((ux > uz ? ux : uz) <= 20) {
            int ox = jbo_osd_pp(c, 0, lx, sx, est);
            int oz = jbo_osd_pp(c, 1, lz, sz, est);
            if (ox || oz) {
                ok = syn_equal(c, 0, est, sx) && syn_equal(c, 1, est, sz);
                if (ok) osd_ok = 1;
            }
        }
    }
    int exact = memcmp(est, err, n) == 0, stab = 0, success = ok;
    if (ok) {
        int words = (n + 63) / 64;
        uint64_t *dx = (uint64_t *)calloc(words, 8), *dz = (uint64_t *)calloc(words, 8);
        for (int i = 0; i < n; ++i) {
            if (xbit(err[i]) ^ xbit(est[i])) dx[i >> 6] |= 1ull << (i & 63);
            if (zbit(err[i]) ^ zbit(est[i])) dz[i >> 6] |= 1ull << (i & 63);
        }
        stab = jbo_in_row_space(bz, dx) && jbo_in_row_space(bx, dz);
        success = ok && stab;
        free(dx); free(dz);
    }
    memset(rec, 0, sizeof(*rec));
    rec->trial_idx = trial_idx;
    rec->iterations = r.iterations;
    rec->bp_ok = r.bp_ok;
    rec->syndrome_ok = ok;
    rec->success = success;
    rec->exact = exact;
    rec->stab_equiv = stab;
    rec->pp_in_decode = r.pp_success;
    rec->pp_in_ets = r.pp_success_ets;
    rec->pp_in_flip = r.pp_success_flip;
    rec->ets_pp_ok = ets_ok;
    rec->flip_pp_ok = flip_ok;
    rec->osd_pp_ok = osd_ok;
    rec->used_any = used_any;
    rec->used6 = used6;
    rec->used12 = used12;
    rec->ets_applied_post = ets_applied;
    rec->pp_success_this = success && (r.pp_success || ets_ok || flip_ok || osd_ok);
    rec->osd_success = osd_ok || (r.pp_success && !r.pp_success_ets && !r.pp_success_flip);
    if (est_out) memcpy(est_out, est, n);
    free(err); free(est); free(sx); free(sz); free(lx); free(lz);
    return 0;
}

/* Sampled trial (5931-5946) followed by jbo_error_trial. */
int jbo_simulate_trial(const jbo_code *c, const jbo_ets_set *ets, const jbo_basis *bx, const jbo_basis *bz,
                       jbo_work *w, uint64_t seed, long long trial_idx, double p, int max_iter, int flip_hist,
                       double damping, int freeze_syn, int enable_pp, jbo_trial_record *rec, uint8_t *err_out,
                       uint8_t *est_out) {
    uint8_t *err = (uint8_t *)malloc(c->n);
    jbo_sample(seed, trial_idx, p, c->n, err);
    int rc = jbo_error_trial(c, ets, bx, bz, w, err, trial_idx, p, max_iter, flip_hist, damping, freeze_syn, enable_pp,
                             rec, est_out);
    if (err_out) memcpy(err_out, err, c->n);
    free(err);
    return rc;
}

int jbo_wilson(long long n, long long k, double z, double *lo, double *hi) {
    if (n <= 0) return 0;
    double nn = (double)n, ph = (double)k / nn, z2 = z * z;
    double den = 1.0 + z2 / nn;
    double center = (ph + z2 / (2.0 * nn)) / den;
    double half = z * sqrt((ph * (1.0 - ph) + z2 / (4.0 * nn)) / nn) / den;
    *lo = center - half > 0.0 ? center - half : 0.0;
    *hi = center + half < 1.0 ? center + half : 1.0;
    return 1;
}
