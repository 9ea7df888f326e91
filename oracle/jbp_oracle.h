/* CPU oracle for the joint X/Z BP + post-processing Monte-Carlo path (test infrastructure).
 *
 * A plain-C restatement of the reference decoder in jointbp_ets.cpp, written from its
 * behaviour: same messages, same floating-point operation order (no FMA contraction),
 * same decision rules.  It is the checker for the CUDA kernels: only tests, the bench's
 * CPU-baseline leg and the smoke check may load it.  It is pinned against the reference
 * itself (oracle/_ref, built from the reference sources) by tests/test_oracle_pin.py.
 *
 * Pauli states: 0=I, 1=X, 2=Z, 3=Y.  Side 0 = X checks (test x-bits), side 1 = Z checks.
 */
#ifndef JBP_ORACLE_H
#define JBP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;             /* variables (qubits) */
    int m[2];          /* checks per side */
    int e[2];          /* edges per side */
    int P;             /* circulant size of the APM construction (ETS token decoding), 0 if none */
    int *chk_off[2];   /* m+1 CSR offsets; edge id = chk_off[c] + position */
    int *chk_var[2];   /* variable of each edge, check-major */
    int *var_off[2];   /* n+1 offsets into var_edge */
    int *var_edge[2];  /* edges of each variable, ascending check index */
} jbo_code;

/* ETS table of one size and side (jointbp_ets.cpp:3114-3123). */
typedef struct {
    int var_count;     /* variables per entry (<= 32) */
    int count;         /* entries, in file order */
    int *vars;         /* count * var_count, each entry sorted ascending */
    uint64_t *key;     /* (c0 << 32) | c1 of the sorted unsatisfied pair */
} jbo_ets;

#define JBO_MAX_ETS_GROUPS 16
typedef struct {
    int ngroups;
    int size[JBO_MAX_ETS_GROUPS];
    char label[JBO_MAX_ETS_GROUPS][8];
    int loaded[JBO_MAX_ETS_GROUPS][2];
    jbo_ets tab[JBO_MAX_ETS_GROUPS][2];
} jbo_ets_set;

typedef struct {
    int words;         /* 64-bit words per row */
    int rank;
    uint64_t *rows;    /* rank * words */
    int *pivot;        /* highest set bit of each row */
    int *order;        /* rows by descending pivot */
} jbo_basis;

typedef struct {
    int iterations;
    int syndrome_ok;       /* est reproduces the target syndrome */
    int bp_ok;             /* converged by plain BP */
    int pp_success;        /* in-loop PP succeeded */
    int pp_success_ets;
    int pp_success_flip;
    int pp_used_ets_any;
    int pp_used_ets6;
    int pp_used_ets12;
    unsigned ets_label_mask; /* bit g set when ETS group g was applied in the in-loop success */
} jbo_result;

/* Per-trial Monte-Carlo record (same fields as the reference harness). */
typedef struct {
    long long trial_idx;
    int iterations, bp_ok, syndrome_ok, success, exact, stab_equiv;
    int pp_in_decode, pp_in_ets, pp_in_flip;
    int ets_pp_ok, flip_pp_ok, osd_pp_ok;
    int used_any, used6, used12, ets_applied_post, pp_success_this, osd_success;
} jbo_trial_record;

/* Decoder scratch and side outputs; allocate with jbo_work_new. */
typedef struct jbo_work jbo_work;

int jbo_code_from_params(const char *path, jbo_code *out);
int jbo_code_from_checks(int n, int mx, const int *xoff, const int *xvar, int mz, const int *zoff,
                         const int *zvar, jbo_code *out);
void jbo_code_free(jbo_code *c);

void jbo_syndrome(const jbo_code *c, int side, const uint8_t *err, uint8_t *syn);

uint64_t jbo_trial_seed(uint64_t base_seed, uint64_t trial_idx);
void jbo_sample(uint64_t base_seed, long long trial_idx, double p, int n, uint8_t *err);

int jbo_basis_build(const jbo_code *c, int side, jbo_basis *out);
void jbo_basis_free(jbo_basis *b);
int jbo_in_row_space(const jbo_basis *b, uint64_t *vec);

int jbo_ets_load(const char *path, int P, int expected_vars, char side, jbo_ets *out);
int jbo_ets_set_load_dir(const char *dir, int P, jbo_ets_set *out);
void jbo_ets_set_free(jbo_ets_set *s);
/* Group g of a loaded set: size, label (8 bytes) and entry counts per side; returns ngroups. */
int jbo_ets_info(const jbo_ets_set *s, int g, int *size, char *label, int *count_x, int *count_z);

jbo_work *jbo_work_new(const jbo_code *c);
void jbo_work_free(jbo_work *w);

/* Joint BP with optional in-loop PP.  est (n bytes) receives the estimate.  When
 * abs_llr_x/z are non-null they receive the |LLR| of the last computed iteration
 * (collected every iteration when PP is on, otherwise on iteration max_iter only). */
int jbo_decode(const jbo_code *c, const jbo_ets_set *ets, jbo_work *w, const uint8_t *sx, const uint8_t *sz,
               double p, int max_iter, int flip_hist, int freeze_syn, double damping, int enable_pp,
               uint8_t *est, double *abs_llr_x, double *abs_llr_z, jbo_result *res);

/* Post-BP stages on a final estimate (jointbp_ets.cpp:6020-6197), applied in place. */
int jbo_ets_fix_multi(const jbo_code *c, const jbo_ets_set *ets, int side, const uint8_t *target, uint8_t *est,
                      int *applied_size, int *applied_group);
int jbo_flip_pp(const jbo_code *c, int side, const int *vars, int nv, const uint8_t *target, uint8_t *est);
int jbo_osd_pp(const jbo_code *c, int side, const double *abs_llr, const uint8_t *target, uint8_t *est);

/* Trial body from a known error (syndrome, decode, post-BP PP, classification). */
int jbo_error_trial(const jbo_code *c, const jbo_ets_set *ets, const jbo_basis *bx, const jbo_basis *bz,
                    jbo_work *w, const uint8_t *err, long long trial_idx, double p, int max_iter, int flip_hist,
                    double damping, int freeze_syn, int enable_pp, jbo_trial_record *rec, uint8_t *est_out);

/* Full trial (sample, decode, post-BP PP, classification) like the reference simulate loop. */
int jbo_simulate_trial(const jbo_code *c, const jbo_ets_set *ets, const jbo_basis *bx, const jbo_basis *bz,
                       jbo_work *w, uint64_t seed, long long trial_idx, double p, int max_iter, int flip_hist,
                       double damping, int freeze_syn, int enable_pp, jbo_trial_record *rec, uint8_t *err_out,
                       uint8_t *est_out);

/* Wilson score interval (jointbp_ets.cpp:4388-4399). */
int jbo_wilson(long long n, long long k, double z, double *lo, double *hi);

#ifdef __cplusplus
}
#endif
#endif
