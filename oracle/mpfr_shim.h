/* mpfr_shim.h -- ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Hand-written declarations of the handful of public GMP 6.3 / MPFR 4.2.1 /
 * MPC 1.3.1 entry points the oracle needs.  The system runtime libraries
 * (libmpfr.so.6, libmpc.so.3, libgmp.so.10) are present in this image but their
 * development headers are not, so the oracle links the shared objects by full
 * path and declares the public ABI itself.  Only documented public types and
 * functions appear here (MPFR manual "Custom Interface", "Basic Arithmetic
 * Functions", mpfr_dot/mpfr_sum; MPC manual "Basic Arithmetic").
 *
 * Layout facts relied upon (LP64, public in mpfr.h / mpc.h):
 *   __mpfr_struct = { long prec; int sign; long exp; mp_limb_t *d; }
 *   __mpc_struct  = { __mpfr_struct re[1]; __mpfr_struct im[1]; }
 *   MPFR_RNDN = 0, MPC_RNDNN = MPC_RND(MPFR_RNDN, MPFR_RNDN) = 0.
 * A regular MPFR number equals 0.d * 2^exp with the most significant bit of
 * d[ceil(prec/64)-1] set and the low (64*limbs - prec) bits zero, which is the
 * same significand/exponent convention as cu_fp::cu_freal<PB>.
 */
#ifndef MPB_ORACLE_MPFR_SHIM_H
#define MPB_ORACLE_MPFR_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long shim_limb_t;
typedef long shim_prec_t;
typedef long shim_exp_t;
typedef int shim_rnd_t;

typedef struct {
  shim_prec_t prec;
  int sign;
  shim_exp_t exp;
  shim_limb_t *d;
} shim_mpfr_struct;
typedef shim_mpfr_struct shim_mpfr_t[1];
typedef shim_mpfr_struct *shim_mpfr_ptr;

typedef struct {
  shim_mpfr_struct re[1];
  shim_mpfr_struct im[1];
} shim_mpc_struct;
typedef shim_mpc_struct shim_mpc_t[1];
typedef shim_mpc_struct *shim_mpc_ptr;

#define SHIM_RNDN 0
#define SHIM_MPC_RNDNN 0

/* MPFR custom-interface kinds (mpfr.h: MPFR_NAN_KIND..MPFR_REGULAR_KIND) */
#define SHIM_ZERO_KIND 2
#define SHIM_REGULAR_KIND 3

/* ---- MPFR ---- */
const char *mpfr_get_version(void);
void mpfr_init2(shim_mpfr_ptr, shim_prec_t);
void mpfr_clear(shim_mpfr_ptr);
void mpfr_set_prec(shim_mpfr_ptr, shim_prec_t);
void mpfr_custom_init_set(shim_mpfr_ptr, int kind, shim_exp_t, shim_prec_t, void *);
int mpfr_set(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
void mpfr_set_zero(shim_mpfr_ptr, int);
int mpfr_zero_p(const shim_mpfr_struct *);
int mpfr_equal_p(const shim_mpfr_struct *, const shim_mpfr_struct *);
int mpfr_signbit(const shim_mpfr_struct *);
int mpfr_mul(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_add(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_sub(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_div(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_sqrt(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_exp(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_log(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_expm1(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_log1p(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_sin(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_cos(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_tan(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_atan(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_sinh(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_cosh(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_atanh(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_asin(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_acos(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_cbrt(shim_mpfr_ptr, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_pow(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_atan2(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_div_ui(shim_mpfr_ptr, const shim_mpfr_struct *, unsigned long, shim_rnd_t);
int mpfr_const_pi(shim_mpfr_ptr, shim_rnd_t);
int mpfr_const_log2(shim_mpfr_ptr, shim_rnd_t);
int mpfr_fma(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *,
             const shim_mpfr_struct *, shim_rnd_t);
int mpfr_fmms(shim_mpfr_ptr, const shim_mpfr_struct *, const shim_mpfr_struct *,
              const shim_mpfr_struct *, const shim_mpfr_struct *, shim_rnd_t);
int mpfr_dot(shim_mpfr_ptr, const shim_mpfr_ptr *, const shim_mpfr_ptr *,
             unsigned long, shim_rnd_t);
int mpfr_sum(shim_mpfr_ptr, const shim_mpfr_ptr *, unsigned long, shim_rnd_t);
double mpfr_get_d(const shim_mpfr_struct *, shim_rnd_t);
int mpfr_set_d(shim_mpfr_ptr, double, shim_rnd_t);

/* ---- MPC ---- */
const char *mpc_get_version(void);
void mpc_init2(shim_mpc_ptr, shim_prec_t);
void mpc_clear(shim_mpc_ptr);
int mpc_mul(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *, int);
int mpc_add(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *, int);
int mpc_sub(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *, int);
int mpc_fma(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *,
            const shim_mpc_struct *, int);
int mpc_dot(shim_mpc_ptr, const shim_mpc_ptr *, const shim_mpc_ptr *, unsigned long, int);
int mpc_cmp(const shim_mpc_struct *, const shim_mpc_struct *);
int mpc_div(shim_mpc_ptr, const shim_mpc_struct *, const shim_mpc_struct *, int);
int mpc_exp(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_log(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_sqrt(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_sin(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_cos(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_tan(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_sinh(shim_mpc_ptr, const shim_mpc_struct *, int);
int mpc_cosh(shim_mpc_ptr, const shim_mpc_struct *, int);

#ifdef __cplusplus
}
#endif
#endif /* MPB_ORACLE_MPFR_SHIM_H */
