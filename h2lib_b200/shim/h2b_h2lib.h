/* h2b_h2lib — H2Lib's own bem3d / h2matrix / krylovsolvers entry points backed by the B200 library.
 *
 * Linking libh2b_h2lib_{real,complex}.so in front of H2Lib (the shim first on the link line, or
 * loaded first) makes an unchanged H2Lib program run the hot path on the GPU: the shim defines the
 * same symbols as H2Lib, so the dynamic linker binds the program's calls, and H2Lib's calls among
 * its own functions, to the shim.  The shim records what each H2Lib object is, does the work
 * through include/h2b200.h, writes the results into H2Lib's own host structures, and calls the
 * original H2Lib function (looked up with dlsym(RTLD_NEXT)) for the bookkeeping it leaves to
 * H2Lib.  Which functions are replaced, and the H2Lib interface each one keeps:
 *
 *   new_{slp,dlp,adlp}_laplace_bem3d     Library/laplacebem3d.h:64/93/124  (real build)
 *   new_{slp,dlp,adlp}_helmholtz_bem3d   Library/helmholtzbem3d.h:82/113/145 (complex build)
 *       H2Lib's constructor, then bem->nearfield is set to the GPU block fill (the plugin point
 *       of Library/bem3d.h:380), so every H2Lib driver that fills nearfield blocks uses the GPU.
 *   setup_h2matrix_aprx_inter_bem3d      Library/bem3d.h:2773   records the interpolation order
 *   assemble_bem3d_amatrix               Library/bem3d.h:3029   dense matrix in one launch
 *   assemble_bem3d_h2matrix_row_clusterbasis / _col_clusterbasis   Library/bem3d.h:3160/3188
 *   assemble_bem3d_h2matrix / _nearfield_h2matrix / _farfield_h2matrix  Library/bem3d.h:3216-3258
 *       all blocks of the matrix in one launch per phase; the device matrix stays resident
 *   addeval_h2matrix_avector             Library/h2matrix.h:546  on the resident device matrix
 *   solve_gmres_h2matrix_avector         Library/krylovsolvers.h:299  device GMRES
 *   solve_gmres_avector                  Library/krylovsolvers.h:235  device GMRES when the
 *       operator is addeval_h2matrix_avector on a resident matrix
 *   del_h2matrix, del_laplace_bem3d, del_helmholtz_bem3d, del_surface3d   release device objects
 *
 * Objects the shim did not create on the device are left to H2Lib: an operator of the other
 * field type (Laplace in a USE_COMPLEX build, Helmholtz in a real one) or an H2 matrix that was
 * not assembled through the shim (built by H2Lib's compression routines, say) keeps H2Lib's own
 * code for every call.  Device failures abort with a message, as H2Lib does on its own errors
 * (Library/basic.c:106-117).  A matrix assembled through the shim is treated as unchanged by the
 * program afterwards: products and solves read the device copy.
 */
#ifndef H2B_H2LIB_H
#define H2B_H2LIB_H

#ifdef __cplusplus
extern "C" {
#endif

/* 1: every replaced function calls H2Lib's original instead (for comparisons); 0: the default. */
void h2b_shim_set_bypass(int on);

/* Work done on the device since the program started: [0] nearfield block fills through the
 * callback, [1] dense matrices, [2] cluster bases, [3] H2 matrix assemblies, [4] matrix-vector
 * products, [5] GMRES solves. */
void h2b_shim_counts(unsigned long long out[6]);

#ifdef __cplusplus
}
#endif

#endif
