/* wrt_oracle.h -- FP64 CPU restatement of the reference's grid-sampled 3D
 * Radon / ray transform hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: the tests, the smoke check
 * and the benchmark's CPU-baseline leg call it to check the CUDA library.  The
 * product (libwrt.so and the drop-in programs) never links or calls it.
 *
 * Every function restates one reference function, keeping its arithmetic in
 * the same order so that, compiled the same way (gcc -O2, no FMA contraction),
 * it reproduces the reference's FP64 results bit for bit.  The pins live in
 * tests/test_oracle_pins.py, which compares this library with the
 * reference's own sources compiled into oracle/_ref/ and with the golden
 * fixtures under tests/golden/.
 *
 * Layouts (all flat, row-major, as the reference's text files order them):
 *   volume  v[(ix*n + iy)*n + iz]          x slowest, z fastest
 *   radon   R[(is*nphi + iphi)*ntheta + it] shift, phi, theta (theta fastest)
 *   rays    P[(iz*nshift + is)*nphi + iphi] z-slice, shift, phi (phi fastest)
 *   adjoint A[(iz*n + ix)*n + iy]          z slowest, y fastest
 */
#ifndef WRT_ORACLE_H
#define WRT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SAMPLER_NEAREST = 0, ORC_SAMPLER_TRILINEAR = 1 };

/* radon_grid/src/init.c:165-189 (theta weights as in
 * radon_inversion/backprojection/C/src/init.c:222-249).  theta_w may be NULL. */
void orc_radon_grid_init(int nphi, int ntheta, int nshift, double *phi,
                         double *theta, double *theta_w, double *shift);
/* ray_grid/src/init.c:214-228 */
void orc_ray_grid_init(int nshift, int nphi, double *shift, double *phi);
/* Gauss-Legendre nodes (ascending) and weights on [-1,1]. */
int orc_gauss_legendre(int n, double *x, double *w);

/* radon_grid/src/interp.c:63-87 (nearest "cell" value, cell 2/n). */
double orc_zero_interp(const double *v, int n, double x, double y, double z);
/* radon_grid/src/interp.c:25-60 == ray_grid/src/interp.c:25-60. */
double orc_trilinear(const double *v, int n, double x, double y, double z);

/* radon_grid/src/integral.c:26-58 with the lattice half-extent L as a
 * parameter (the reference hard-codes L = 2n, i.e. nsize/2 with nsize = 4n)
 * and the sampler as a parameter (the reference calls zero_interp). */
double orc_plane_integral(const double *v, int n, double phi, double theta,
                          double shift, int sampler, int half_extent);
/* The radon_grid program's loop nest (radon_grid/src/radon_grid.c:248-259):
 * out[(is*nphi+iphi)*ntheta+it]. */
void orc_radon_forward(const double *v, int n, int nphi, int ntheta, int nshift,
                       int sampler, int half_extent, double *out, int nthreads);
/* Same integral on an explicit list of planes (phi[k], theta[k], shift[k]). */
void orc_radon_planes(const double *v, int n, int nplanes, const double *phi,
                      const double *theta, const double *shift, int sampler,
                      int half_extent, double *out, int nthreads);

/* ray_grid/src/integral.c:11-50.  frame (row-major 3x3, may be NULL for the
 * reference's z-slice frame) rotates the sample points: x_world = F x_local. */
double orc_ray_transform(const double *v, int n, double z, double s,
                         double phi, const double *frame);
/* ray_grid/src/ray_grid.c:243-258 loop nest: out[(iz*nshift+is)*nphi+iphi]. */
void orc_ray_forward(const double *v, int n, int nslices, int nshift, int nphi,
                     const double *frame, double *out, int nthreads);

/* radon_reduction/slicing.c:5-119 and reduction.c:546-563.
 * rays in file order [ngrid][nshift_ray][nphi] (z-slices == ngrid);
 * out[(is*nphi+iphi)*ntheta+it] on the Radon grid (nshift, nphi, ntheta).
 * With nshift == nshift_ray this is exactly the reference; a different
 * nshift decouples the Radon shift grid from the ray offset grid. */
void orc_reduction_forward(const double *rays, int ngrid, int nshift_ray,
                           int nphi, int nshift, int ntheta, double *out,
                           int nthreads);
/* Same on an explicit list of Radon grid indices (is, iphi, it). */
void orc_reduction_planes(const double *rays, int ngrid, int nshift_ray,
                          int nphi, int nshift, int ntheta, int nplanes,
                          const int *is, const int *iphi, const int *it,
                          double *out, int nthreads);

/* radon_inversion/backprojection/C/src/integral.c:6-24 with
 * interp.c:5-28, loop nest radon3d_ajoint.c:240-254.
 * radon in file order [nshift][nphi][ntheta]; out[(iz*n+ix)*n+iy]. */
void orc_adjoint_forward(const double *radon, int nphi, int ntheta, int nshift,
                         int n, double *out, int nthreads);
/* Same at explicit points (x[k], y[k], z[k]). */
void orc_adjoint_points(const double *radon, int nphi, int ntheta, int nshift,
                        int npts, const double *x, const double *y,
                        const double *z, double *out, int nthreads);

/* Exact transpose of orc_radon_forward (same lattice and sampler): adds
 * g[plane] * (sampling weight) into vol_out for every lattice sample.
 * vol_out must be zeroed by the caller. */
void orc_radon_transpose(const double *g, int n, int nphi, int ntheta,
                         int nshift, int sampler, int half_extent,
                         double *vol_out);

#ifdef __cplusplus
}
#endif
#endif
