/*
 * ssenss_gpu_shim.h -- the SSENSS host's side of the binding to
 * libssenss_b200 (ssenss_gpu_shim.c).
 *
 * The shim defines the reference's own solve-path functions (same names,
 * same signatures as src/solver.h, src/global.h, src/poisson.h,
 * src/precon.h, src/convection.h and src/particles.h declare them) and runs
 * them on the GPU through include/ssenss_b200.h.  Besides those it adds the
 * three functions below, which the host calls itself: attach once where
 * initialise_preconditioners(sel) ran (src/main.c:78-79), detach before the
 * elements are freed.
 *
 * Compile with the reference's headers on the include path (it needs
 * struct element and friends) and with include/ of this library.
 */
#ifndef SSENSS_GPU_SHIM_H
#define SSENSS_GPU_SHIM_H

#include "structs.h"

/* Hand the reference's discretisation to the library: the neighbour ids
 * of every element, the stored GLL bases, derivative and interpolation
 * matrices and geometric factors of every p-multigrid level, the
 * dealiasing grid and the particle walk's factors.  One rank only
 * (MPI reduced to a single process).  Returns 0; on failure it calls the
 * reference's fatal_error, as the reference does on every error. */
int ssenss_gpu_attach(struct element **sel, int device);

/* Free the library's context (device memory, stream). */
void ssenss_gpu_detach(void);

/* Outcome of the most recent solve the shim ran (the reference's void
 * solve functions return nothing, so the shim keeps it here): kind 0 =
 * Poisson (flexible CG + p-multigrid), 1 = Helmholtz (Jacobi CG), 2 =
 * conjugate_gradient called directly; status is an ssg_status
 * (SSG_MAXITER when the iteration cap was reached, which the reference
 * also accepts silently).  *history points at sqrt((r.r)_w) after each
 * outer iteration, history_len values. */
struct ssenss_gpu_solve {
	int kind;
	int var;
	int status;
	int iterations;
	double eps;
	double residual;
	double solve_ms;
	int history_len;
	const double *history;
};
const struct ssenss_gpu_solve *ssenss_gpu_last_solve(void);

/* integrate_navier_stokes runs the whole step on the device (on, the
 * default: ssg_navier_stokes_step on the state copied in and out) or the
 * reference's own step with its solves and convection calls bound to the
 * library (off). */
void ssenss_gpu_device_step(int on);

/* The solves of the last integrate_navier_stokes that ran on the device
 * (the pressure solve, then the three velocity solves): *solves points at
 * them; returns how many (0 after a step the reference's code ran). */
int ssenss_gpu_step_solves(const struct ssenss_gpu_solve **solves);

/* the reference's own step, renamed at build time (-Dintegrate_navier_
 * stokes=host_integrate_navier_stokes on src/navier_stokes.c) */
void host_integrate_navier_stokes(struct element **sel);

#endif
