// Serving path: asynchronous commit requests admitted by free HBM budget and
// run concurrently on the context's streams, queued ones admitted together
// as groups that share their launches (continuous batching).
#pragma once
#include "runtime.h"

namespace pico {

pico_status serving_start(pico_ctx* ctx);
void serving_stop(pico_ctx* ctx);

}  // namespace pico
