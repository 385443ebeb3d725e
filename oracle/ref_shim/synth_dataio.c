/*
 * Replacement for the five entry points of src/dataio.c (HDF5 is not in this
 * image).  Test infrastructure: it feeds the unmodified reference sources a
 * mesh held in memory instead of an HDF5 grid file.
 *
 * The grid record is the one src/dataio.c:34-62 and misc/rectangular_grid.py
 * describe: per element 8 trilinear vertices (an n=2 GLL element, i fastest),
 * 6 face, 12 edge and 8 corner neighbour ids (negative = wall code), edge and
 * corner sizes and zero face rotations.  read_grid() maps the vertices to the
 * run's GLL grid by the same interpolation as copy_grid_from_struct
 * (src/dataio.c:407-452), then computes the geometric factors as read_grid does
 * (src/dataio.c:197-227).
 */
#include <stdlib.h>
#include <string.h>
#include "structs.h"
#include "utils.h"
#include "linalg.h"
#include "tripalg.h"
#include "basis.h"
#include "interpolation.h"
#include "geometry.h"
#include "dataio.h"
#include "synth_dataio.h"

struct synth_mesh ssgref_mesh;

void write_log(struct element **sel)
{
	(void) sel;
}

void write_to_file(struct element **sel, const char *filename, int write_data)
{
	(void) sel;
	(void) filename;
	(void) write_data;
}

/* src/dataio.c:150-178 reads U/V/W; here the velocity comes from the
 * harness's buffer (or is zero, as examples/init.h5 is). */
void read_velocity(struct element **sel, const char *filename)
{
	(void) filename;
	const size_t ntot = (*sel)->ntot;
	for (int e = 0; e < (*sel)->nel; ++e)
		for (int c = 0; c < 3; ++c) {
			double *dst = ***sel[e]->u->ind[c];
			if (ssgref_mesh.init_velocity)
				memcpy(dst, ssgref_mesh.init_velocity +
						((size_t) c * (*sel)->nel + e) * ntot,
						ntot * sizeof(double));
			else
				memset(dst, 0, ntot * sizeof(double));
		}
}

void get_grid_size(struct parameters *params, struct communicator *comm,
		const char *filename)
{
	(void) comm;
	(void) filename;
	params->neltot = ssgref_mesh.nel;
	params->nel = ssgref_mesh.nel;
}

void read_grid(struct geometry **geom, struct communicator *comm,
		struct basis *basis, const char *filename)
{
	(void) comm;
	(void) filename;
	const int nel = ssgref_mesh.nel;
	struct basis *vbasis = new_gll_basis(2);
	struct basis *gbasis = new_gll_basis(basis->n);
	create_interpolation_matrices(vbasis, gbasis);
	double ***vtx = new_3d_array(2, 2, 2);

	for (int e = 0; e < nel; ++e) {
		struct geometry *g = geom[e];
		const int *nb = ssgref_mesh.neigh + 26 * (size_t) e;
		g->id = e;
		for (int f = 0; f < 6; ++f) {
			g->neigh_rot[f] = 0;
			g->neigh_el[f] = nb[f];
			g->neigh_proc[f] = nb[f] < 0 ? nb[f] : 0;
		}
		for (int q = 0; q < 12; ++q) {
			g->neigh_edge_el[q] = nb[6 + q];
			g->neigh_edge_proc[q] = nb[6 + q] < 0 ? nb[6 + q] : 0;
			g->edge_size[q] = nb[6 + q] < 0 ? 0 : 1;
		}
		for (int c = 0; c < 8; ++c) {
			g->neigh_corn_el[c] = nb[18 + c];
			g->neigh_corn_proc[c] = nb[18 + c] < 0 ? nb[18 + c] : 0;
			g->corner_size[c] = nb[18 + c] < 0 ? 0 : 1;
		}
		set_boundary_conditions(g);
		for (int d = 0; d < 3; ++d) {
			memcpy(**vtx, ssgref_mesh.vertices + 24 * (size_t) e
					+ 8 * d, 8 * sizeof(double));
			interpolate_to_grid(gbasis, *g->grid->ind[d], vbasis,
					vtx);
		}
	}
	free_3d_array(vtx);
	free_basis(vbasis);
	free_basis(gbasis);

	for (int e = 0; e < nel; ++e)
		compute_geometry_transformations(geom[e], basis);
}
