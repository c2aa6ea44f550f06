/*
 * Serving interface of the B200 triples engine: a request loop that accepts
 * (T) and (fT) solves of uneven sizes as they arrive and runs them with
 * continuous batching on one GPU.  No counterpart in the reference (its
 * entry points, pt.h, solve one system per call; this loop sits beside
 * them and computes the same energies).
 *
 *  - Admission by device memory: each solve needs a computed footprint
 *    (libpt_footprint: its resident amplitudes, integrals, their padded or
 *    digit-plane copies and its round workspace).  A solve is admitted, in
 *    arrival order, when a block of that size is free in the server's
 *    device pool (allocated once, mem_budget bytes) and fewer than
 *    max_active solves are resident; it leaves the pool when its energy is
 *    complete.
 *  - Continuous batching: the admitted solves' triples run in shared
 *    rounds -- one GEMM launch per kernel variant over the triples of many
 *    solves, one energy-epilogue launch, one reduction -- with the
 *    solves of least remaining work first; a request that arrives while
 *    others run joins the next round.  Rounds replay CUDA graphs captured
 *    once per set of kernel variants (the first round of a set launches
 *    directly and captures).
 *  - Each solve's energy is the same as libpt_plan / libpt_{r,u}{pt,ft}
 *    compute for it alone (per-triple energies in fixed order, summed in
 *    queue order): bitwise, whatever else shares its rounds.
 */
#ifndef LIBPT_PT_SERVE_H
#define LIBPT_PT_SERVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct libpt_server libpt_server;

/* Device bytes a solve takes when served (exact: a sizing pass of the plan
 * with no device work).  kind: 0 rpt, 1 upt, 2 rft, 3 uft; dtype 0 FP64,
 * 1 FP32 inputs; precision LIBPT_PREC_* (| slices << 8); host_inputs: the
 * arguments are host pointers (adds a staging buffer); round_triples: the
 * triples of one round the solve may hold (0: the server's choice).
 * Returns 0 for invalid arguments. */
size_t libpt_footprint(int kind, size_t oa, size_t va, size_t ob, size_t vb,
                       int dtype, int precision, int host_inputs,
                       size_t round_triples);

/* Creates a server with a device pool of mem_budget bytes (0: 90% of the
 * free device memory) and at most max_active resident solves (0: 64). */
int libpt_server_create(size_t mem_budget, int max_active,
                        libpt_server **out);

/* Queues a solve.  args: the pt.h arguments of `kind` in the reference's
 * order (host pointers when host_inputs, else device pointers); they must
 * stay valid and unchanged until libpt_server_inputs_released reports them
 * released (at the latest when libpt_server_wait reports the solve done).
 * *ticket identifies it.  Ownership stays with the caller. */
int libpt_server_submit(libpt_server *s, int kind, size_t oa, size_t va,
                        size_t ob, size_t vb, const void *const *args,
                        int dtype, int precision, int host_inputs,
                        uint64_t *ticket);

/* Waits up to timeout_s seconds (< 0: no limit) for a solve; on completion
 * writes its energy (restricted factor 2 applied, as libpt_rpt returns it)
 * and its latency from submission, and returns its status (LIBPT_OK, or the
 * error that ended it).  LIBPT_ERR_TIMEOUT if it is still running. */
int libpt_server_wait(libpt_server *s, uint64_t ticket, double timeout_s,
                      double *energy, double *latency_s);

/* Cancels a solve.  A queued solve leaves the queue at once; one whose plan
 * is being created, or whose triples are running, gets no further rounds
 * and ends as soon as its rounds in flight retire, returning its block to
 * the pool.  Either way libpt_server_wait then reports LIBPT_ERR_CANCELLED
 * (no energy).  A solve that has already ended keeps its result; returns
 * LIBPT_OK (LIBPT_ERR_ARG for an unknown ticket).  The other solves are not
 * affected: their energies stay bitwise those they have alone. */
int libpt_server_cancel(libpt_server *s, uint64_t ticket);

/* Where an ended solve's latency went, in seconds, times[0..3]: waiting for
 * admission (a block of its footprint in the pool and a resident slot),
 * preparing (plan creation in its block: uploads, operand preparation,
 * slice choice, tuning), waiting for its first round, and running (from its
 * first round's launch to its energy, its rounds interleaved with the other
 * resident solves').  They add up to the latency libpt_server_wait reports.
 * LIBPT_ERR_TIMEOUT if the solve has not ended. */
int libpt_server_solve_times(libpt_server *s, uint64_t ticket,
                             double *times);

/* Non-blocking: *released = 1 once the server no longer reads the solve's
 * arguments (its operands are resident in the pool, or it ended), so the
 * caller may free or reuse them before the solve completes. */
int libpt_server_inputs_released(libpt_server *s, uint64_t ticket,
                                 int *released);

/* Counters of the server's life so far. */
typedef struct {
  uint64_t submitted, completed, failed;
  uint64_t rounds, graph_rounds, triples, launches;
  double flops;              /* reference GEMM flops of the triples run */
  size_t pool_bytes;         /* the device pool */
  size_t bytes_in_use, peak_bytes_in_use;
  uint64_t max_resident;     /* most solves resident at once */
} libpt_server_stats;

int libpt_server_stats_get(libpt_server *s, libpt_server_stats *out);

/* Drains outstanding solves, stops the threads, releases the pool. */
int libpt_server_destroy(libpt_server *s);

#ifdef __cplusplus
}
#endif

#endif
