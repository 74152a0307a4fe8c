/* spiffe_b200_geometry.h -- define_geometry: boundary points to metal flags.
 *
 * Rasterises a POISSON/SUPERFISH-style list of &po boundary points onto the
 * node lattice and derives the per-node field flags, as
 * process_geometry_definition (geometry.c:21-369) with the drawing routines
 * of grid_drawing.c does.  Host code; the result is what spiffe_gpu_create
 * takes as `flags`.
 */
#ifndef SPIFFE_B200_GEOMETRY_H
#define SPIFFE_B200_GEOMETRY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* define_geometry variables (geometry.nl:8-38) that shape the lattice */
typedef struct spiffe_geometry_options {
  int32_t nz, nr;
  double zmin, zmax, rmax;
  double zr_factor; /* boundary coordinates are multiplied by this */
} spiffe_geometry_options;

/* Reads the &po points of `boundary_text` (the contents of the file named by
 * define_geometry's `boundary`) and fills flags and psi_imposed, each
 * (nz+1)*(nr+1) values, ir fastest; material may be NULL.  Returns 0, or a
 * negative code with spiffe_gpu_last_error() describing the problem (points
 * outside the region, malformed points), where the reference exits. */
int spiffe_geometry_rasterise(const spiffe_geometry_options *opt, const char *boundary_text, int16_t *flags,
                              double *psi_imposed, int16_t *material);

/* getBoundaryPoints (grid_drawing.c:541-760), the surface a define_emitter of
 * `material_id` emits from: the nodes of the first run of boundary points of
 * that material (in drawing order, corners inserted so that one index changes
 * at a time) and, per segment k -> k+1, the side it emits to (direction[k],
 * SPIFFE_EMITS_* of spiffe_b200_types.h; the last entry unused).  *n_points is 0 when no boundary
 * point has the material.  With iz, ir and direction all NULL only
 * *n_points is set. */
int spiffe_geometry_boundary_points(const spiffe_geometry_options *opt, const char *boundary_text, int32_t material_id,
                                    int64_t max_points, int32_t *iz, int32_t *ir, int16_t *direction,
                                    int64_t *n_points);

#ifdef __cplusplus
}
#endif

#endif
