/* Single-rank stand-in for the few MPI calls made by the reference engine
 * (dragonfly/src/max_prob.c:55,234,241,260,355-423; max_scale.c:127,279).
 *
 * Test infrastructure only: it lets the reference C sources compile without an
 * MPI installation so that they can serve as a CPU oracle. With one rank every
 * reduction is the identity: a collective with a separate send buffer copies it
 * into the receive buffer, and MPI_IN_PLACE leaves the buffer untouched.
 */
#ifndef DFG_ORACLE_SHIM_MPI_H
#define DFG_ORACLE_SHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_IN_PLACE ((void *)1)

static inline int dfg_shim_copy(const void *src, void *dst, int count, MPI_Datatype t) {
	if (src != MPI_IN_PLACE && src != dst && dst != NULL && count > 0)
		memcpy(dst, src, (size_t)count * (size_t)t);
	return 0;
}

static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
	(void)op; (void)c;
	return dfg_shim_copy(s, r, n, t);
}

static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
	(void)op; (void)root; (void)c;
	return dfg_shim_copy(s, r, n, t);
}

static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
	(void)b; (void)n; (void)t; (void)root; (void)c;
	return 0;
}

/* Rank 0 gathers in place from itself: nothing moves. */
static inline int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rn,
                              const int *displ, MPI_Datatype rt, int root, MPI_Comm c) {
	(void)s; (void)sn; (void)st; (void)r; (void)rn; (void)displ; (void)rt; (void)root; (void)c;
	return 0;
}

#endif
