// Batched decomposition (scc_batch.cu): device counter layout.
#pragma once
#include "scc_internal.cuh"

#define BATCH_CTR_NEXT 0          // next graph to take
#define BATCH_CTR_ERROR 32        // device error code
#define BATCH_CTR_ROUNDS 64       // FW-BW rounds over all graphs
#define BATCH_CTR_LEVELS 65       // reachability levels over all graphs
#define BATCH_CTR_MAX_ROUNDS 66   // most rounds one graph took
#define BATCH_CTR_WORDS 96
