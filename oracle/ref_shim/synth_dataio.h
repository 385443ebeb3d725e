/* In-memory mesh handed to the reference build (test infrastructure). */
#ifndef SSG_REF_SYNTH_DATAIO_H
#define SSG_REF_SYNTH_DATAIO_H

struct synth_mesh {
	int nel;
	const double *vertices;      /* nel x {x[8], y[8], z[8]} */
	const int *neigh;            /* nel x {face[6], edge[12], corner[8]} */
	const double *init_velocity; /* 3 x nel x n^3, or NULL for zero */
};

extern struct synth_mesh ssgref_mesh;

#endif
