/* CPU restatement of hfscf's two-electron algorithms, used as the test oracle.
 *
 * TEST INFRASTRUCTURE ONLY: tests, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py call this library as the checker.  The product never links it.
 *
 * Every function restates the reference file:line given beside it.  Parity of
 * this restatement with the reference itself is pinned by tests that compare it
 * with the reference's own integral code compiled in place (oracle/_ref) and with
 * fixtures generated from that code (tests/golden/).
 *
 * Shell description shared by all entry points (flat arrays):
 *   nshell, L[nshell], xyz[3*nshell] (bohr), nprim[nshell],
 *   alpha[sum nprim], coef[sum nprim] (UNNORMALISED, as in the .gbs file),
 *   pure (1 = spherical functions, 0 = Cartesian).
 */
#ifndef HFSCF_ORACLE_H
#define HFSCF_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

double or_boys(int m, double T);
void or_shell_norm(int L, int nprim, const double* alpha, const double* coef, double* out);
void or_ylm(int L, double* out);
long long or_index_ijkl(long long i, long long j, long long k, long long l);
long long or_packed_len(long long n);
long long or_nbf(int nshell, const int* L, int pure);

int or_eri_packed(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                  const double* coef, int pure, double* eri);
int or_shell_quartet(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
                     const double* coef, int pure, int si, int sj, int sk, int sl, double* block);
int or_fock_rhf(long long n, const double* eri, const double* D, const double* H, double* F);
int or_fock_uhf(long long n, const double* eri, const double* Da, const double* Db, const double* H,
                double* Fa, double* Fb);
int or_jk(long long n, const double* eri, const double* D, double* J, double* K);
int or_jk_packed(long long n, const double* eri, int nd, const double* D, double* J, double* K);
int or_grad2e_from_deriv1(long long n, const double* deriv9, const int* bf_atom, int natoms, const double* DJ,
                          double cJ, int nK, const double* DK, double cK, double* grad);
int or_grad2e(int nshell, const int* L, const double* xyz, const int* nprim, const double* alpha,
              const double* coef, int pure, const int* shell_atom, int natoms, const double* DJ, double cJ,
              int nK, const double* DK, double cK, double* grad);

#ifdef __cplusplus
}
#endif
#endif
