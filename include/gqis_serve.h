/* gqis_serve.h - C ABI of the native sweep server (libgqis_serve.so).
 *
 * No counterpart in the reference, which runs one synchronous launch per mesolve_2D call
 * (gqis/solver.py:2322-2340). The server lets any C/C++ host submit sweeps of any compiled model
 * module (include/gqis_b200.h) while others run: requests are admitted by a device-memory budget
 * and a slot limit, cut into point chunks, and the chunks of different requests run concurrently
 * on several CUDA streams (continuous batching). Each point's result depends only on its own
 * inputs, so a request's results are the same alone and in the mix.
 *
 * The caller owns every request buffer (the descriptor's device pointers); they must stay valid
 * until the request has ended (DONE, FAILED or CANCELLED). The server allocates only its own
 * streams, events and a small array of work counters for adaptive chunks. All functions return
 * a GQIS_* status; gqis_serve_last_error() describes the last failure of the calling thread.
 * A server handle may be used from several host threads. Ended requests stay queryable (state,
 * error text) until gqis_serve_close, a few hundred bytes each.
 */
#ifndef GQIS_SERVE_H
#define GQIS_SERVE_H

#include <stdint.h>

#include "gqis_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* request states */
#define GQIS_REQ_QUEUED 0
#define GQIS_REQ_RUNNING 1
#define GQIS_REQ_DONE 2
#define GQIS_REQ_FAILED 3
#define GQIS_REQ_CANCELLED 4

typedef struct gqis_server gqis_server;

/* Start a server on CUDA device `device` with `streams` streams, at most `max_inflight` admitted
 * requests, chunks of at most `chunk_points` points, and `memory_budget` bytes of request memory
 * (the sum of the admitted requests' stated bytes; 0: no limit). */
int gqis_serve_open(int device, int streams, int max_inflight, int64_t chunk_points, int64_t memory_budget,
                    gqis_server** out);

/* Queue one sweep: the model module at `module_path` (loaded once per server) and a complete
 * descriptor of its launch (device buffers of `device`). `bytes`: the request's device memory for
 * admission (0 if not counted). The request id is written to *request_id. */
int gqis_serve_submit(gqis_server* server, const char* module_path, const gqis_sweep_desc* desc, int64_t bytes,
                      int64_t* request_id);

/* Current state (GQIS_REQ_*) of a request. */
int gqis_serve_poll(gqis_server* server, int64_t request_id, int32_t* state);

/* Wait until the request has ended or `timeout_s` seconds have passed (GQIS_ERR_TIMEOUT). */
int gqis_serve_wait(gqis_server* server, int64_t request_id, double timeout_s, int32_t* state);

/* Cancel a request: a queued one ends at once, a running one after its chunks in flight. */
int gqis_serve_cancel(gqis_server* server, int64_t request_id);

/* Error text of a FAILED request (the module's message of the failing launch) into buf[len]. */
int gqis_serve_request_error(gqis_server* server, int64_t request_id, char* buf, int64_t len);

/* Cancel every request that has not ended (queued ones at once, running ones after their chunks
 * in flight), stop the server thread and free the server's streams, events and counters. No other
 * call on the handle may be in progress (in any thread) or follow: the handle is invalid afterwards. */
int gqis_serve_close(gqis_server* server);

const char* gqis_serve_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GQIS_SERVE_H */
