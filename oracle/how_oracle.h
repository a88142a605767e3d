/* how_oracle.h -- CPU restatement of the HOW-MHD time-step path.
 * TEST INFRASTRUCTURE ONLY: the checker for the B200 path, loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the
 * product.  Parity of this restatement with the reference itself is pinned by
 * tests/test_oracle_pin.py (reference sources built by oracle/Makefile into
 * oracle/_ref/) and by the committed fixtures under tests/golden/.
 *
 * State layout is the reference's: q(stage 0..5, var 0..7, i, j, k) with k
 * fastest and 3 ghost cells per side (src/main.cpp:101-120); face B
 * bxb/byb/bzb(stage, i, j, k) (src/fluxct.cpp:27-35).
 */
#ifndef HOW_ORACLE_H
#define HOW_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;          /* active cells per axis                       */
    int bc[3];               /* 0 = periodic, 1 = open                      */
    double xsize, ysize, zsize;
    double gam, cour, rhomin, pgmin;
} oracle_params;

void*  oracle_create(const oracle_params* p);
void   oracle_destroy(void* h);
int    oracle_init_problem(void* h, const char* name);   /* reference problems */
void   oracle_set_q(void* h, int stage, const double* q);
void   oracle_get_q(void* h, int stage, double* q);
void   oracle_set_faceb(void* h, int stage, const double* bx, const double* by, const double* bz);
void   oracle_get_faceb(void* h, int stage, double* bx, double* by, double* bz);
void   oracle_bound(void* h, int stage);
void   oracle_bound_bfield(void* h, int stage);
void   oracle_init_faceb(void* h);
double oracle_tstep(void* h);
void   oracle_ssprk(void* h, double dt);
/* main-loop semantics (src/main.cpp:158-223); max_steps < 0 = unlimited */
int    oracle_run(void* h, double tend, int nt, long max_steps,
                  double* time_out, long* steps_out, double* dts_out, long dts_cap);
/* stage iw = 1 only: copy, bound, ONE directional sweep (dir 0,1,2) with dt;
 * ct_a/ct_b receive the two CT flux arrays that sweep fills. */
void   oracle_sweep(void* h, int dir, double dt, double* q1_out, double* ct_a, double* ct_b);
/* stage iw = 1 up to its CT: zero the CT arrays, copy q(0) and face B(0)
 * into stage 1, bound q(0), the x/y/z sweeps with dt. */
void   oracle_stage1_sweeps(void* h, double dt);
/* bound_bfield(iw - 1) + fluxct(q, iw, k1, k3) on the CT arrays the last
 * sweeps filled; prot(q, stage); a CT array (0..11 = fsy fsz gsx gsz hsx hsy
 * Ox2 Oy2 Oz2 Ox Oy Oz). */
void   oracle_fluxct(void* h, int iw, double k1, double k3);
void   oracle_prot(void* h, int stage);
void   oracle_get_ct(void* h, int which, double* out);
void   oracle_set_threads(int n);
void   oracle_set_ct_avg(int points);   /* 2 (reference) or 4 */
/* algorithmic FP64 operation counts (add/sub/mul/div/sqrt/max/abs as 1) of the
 * per-cell and per-interface kernels, from a counting scalar type. */
void   oracle_flop_counts(double* out, int cap);

#ifdef __cplusplus
}
#endif
#endif
