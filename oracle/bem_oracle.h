/*
 * bem_oracle.h -- CPU FP64 restatement of the BEM-MECECCS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it.  The product path (libbem_b200.so) never links or calls it.
 *
 * Every routine restates one routine of the reference Fortran program
 * (giulianobelinassi/BEM-MECECCS, src/), cited per function.  Arrays keep the
 * reference's Fortran column-major layouts:
 *   cone[k*n + i]          CONE(i+1,k+1), 1-based node numbers, n x 4
 *   etas[3*j + c]          ETAS(c+1,j+1)
 *   hestdiag[9*a + 3*j + i] HESTdiag(i+1,j+1,a+1)
 *   zh[col*nn + row]       ZH(row+1,col+1), complex as interleaved (re,im)
 *
 * Status codes: 0 = ok, 1 = degenerate Jacobian (DET < 1e-5; the reference
 * STOPs, Nonsinge.for:88-96, Nonsingd.for:89-95), 2 = singular matrix.
 */
#ifndef BEM_ORACLE_H
#define BEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

int orc_version(void);

/* Gauleg.for:9-36: NPG-point Gauss-Legendre rule on [-1,1]. */
void orc_gauleg(int npg, double *gi, double *ome);

/* Normvec.for:4-39: unit normal (P2-P1)x(P3-P1) per element. */
void orc_normvec(int n, const int *cone, const double *cx, const double *cy,
                 const double *cz, double *etas);

/* Inputece.for:100-102: collocation point = mean of the 4 nodes. */
void orc_centroids(int n, const int *cone, const double *cx, const double *cy,
                   const double *cz, double *cxm, double *cym, double *czm);

/* Inputecd.for:58-60: complex shear modulus and wave speeds. */
void orc_material(double ge, double rnu, double dam, double rho,
                  double *zge, double *zcs, double *zcp);

/* Ghmatece.for:55-63: static constants C1..C4 (c[0..3]). */
void orc_static_consts(double rmu, double rnu, double *c);

/* Ghmatece.for:92-183 (+ RIGID_BODY :258-282, GEST_SINGULAR :288-323).
 * hest (3nbe x 3n, column-major) may be NULL. */
int orc_ghmatece(int n, int nbe, int np, int npg, const int *cone,
                 const double *cx, const double *cy, const double *cz,
                 const double *cxm, const double *cym, const double *czm,
                 const double *etas, const double *gi, const double *ome,
                 double rmu, double rnu, double *hestdiag, double *gestdiag,
                 double *hest);

/* Ghmatecd.for:113-166: dynamic ZH, ZG before the boundary-condition swap. */
int orc_ghmatecd(int n, int nbe, int np, int npg, const int *cone,
                 const double *cx, const double *cy, const double *cz,
                 const double *cxm, const double *cym, const double *czm,
                 const double *etas, const double *gi, const double *ome,
                 const double *c, const double *zge, const double *zcs,
                 const double *zcp, double fr, const double *hestdiag,
                 const double *gestdiag, double *zh, double *zg);

/* The same for element columns jlo..jhi-1 only (a bounded sample). */
int orc_ghmatecd_cols(int n, int nbe, int np, int npg, const int *cone,
                      const double *cx, const double *cy, const double *cz,
                      const double *cxm, const double *cym, const double *czm,
                      const double *etas, const double *gi, const double *ome,
                      const double *c, const double *zge, const double *zcs,
                      const double *zcp, double fr, const double *hestdiag,
                      const double *gestdiag, int jlo, int jhi, double *zh,
                      double *zg);

/* Ghmatecd.for:316-333 as called at :168 (effective semantics:
 * column j with KODE=0: ZH(:,j) <- -ZG(:,j); ZG(:,j) <- -ZH(:,j)*ZGE). */
void orc_boundary_conditions(int nn, double *zh, double *zg, const int *kode,
                             const double *zge);

/* Ghmatecd.for:172-181: ZFI = ZG * ZDFI (ZGEMV 'N'). */
void orc_zgemv(int nn, const double *a, const double *x, double *y);

/* LAPACK ZGESV (Linsolve.for:94-100), restated: right-looking LU with
 * partial pivoting (IZAMAX |re|+|im|, first maximum), unit lower L, then
 * ZGETRS.  a is overwritten by L\U, b by the solution; ipiv 1-based. */
int orc_zgesv(int nn, double *a, int *ipiv, double *b);

/* Interec.for:59-67: un-swap ZFI/ZDFI for KODE=0 entries. */
void orc_unswap(int nn, const int *kode, const double *zge, double *zfi,
                double *zdfi);

/* EXTENSION, no reference counterpart: the static boundary solve from the
 * reference's static pieces (H: NONSINGE + HESTdiag; G: NONSINGE_G +
 * GESTdiag), the boundary-condition swap with real GE, G*DFI, ZGESV and the
 * un-swap.  disp/trac: 3nbe real; h_out/g_out (nn x nn) may be NULL. */
int orc_static_solve(int n, int nbe, int np, int npg, const int *cone,
                     const double *cx, const double *cy, const double *cz,
                     const double *cxm, const double *cym, const double *czm,
                     const double *etas, const double *gi, const double *ome,
                     double ge, double rnu, const int *kode, const double *dfi,
                     double *disp, double *trac, double *h_out, double *g_out);

/* Interec.for:81-139: interior displacements ZDSOL(3L). */
int orc_interior_disp(int n, int nbe, int np, int npg, const int *cone,
                      const double *cx, const double *cy, const double *cz,
                      const double *etas, const double *gi, const double *ome,
                      int l, const double *cxi, const double *cyi,
                      const double *czi, const double *zge, const double *zcs,
                      const double *zcp, double fr, const double *zfi,
                      const double *zdfi, double *zdsol);

/* Interec.for:186-285 + Sigmaec.for:9-212: interior stresses ZSSOL(9L). */
int orc_interior_stress(int n, int nbe, int np, int npg, const int *cone,
                        const double *cx, const double *cy, const double *cz,
                        const double *etas, const double *gi,
                        const double *ome, int l, const double *cxi,
                        const double *cyi, const double *czi,
                        const double *zge, const double *zcs,
                        const double *zcp, double rho, double fr,
                        const double *zfi, const double *zdfi, double *zssol);

/* Solfund.for:18-60 at one point, for unit checks: zu, zt are 3x3 complex
 * column-major (ZU(i,j) at zu[2*(3*j+i)]). */
void orc_solfund(const double *p, const double *g, const double *rn,
                 const double *zge, const double *zcs, const double *zcp,
                 double fr, double *zu, double *zt);

#ifdef __cplusplus
}
#endif
#endif
