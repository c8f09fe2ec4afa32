// Definition of the single-instance context shared by the C-ABI sources.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "lh_engine.h"

struct lh_ctx {
    lh::DevInstance dev;
    lh::Plan plan;
    lh::Inst *d_inst = nullptr;
    cudaStream_t st = nullptr;
    int device = 0;            // the CUDA device current at lh_ctx_create
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool have_state = false;
    double *d_spec = nullptr;  // spectra accumulators (lh_diag.cu), allocated on first use
    int spec_count = 0;        // accumulations since the last reset
    double *d_stats = nullptr; // stats accumulators (lh_diag.cu), allocated on first use
    int stats_count = 0;
    lh::StatsScratch stats_scr;  // stats transform scratch and pressure snapshot
    std::string err;
};
