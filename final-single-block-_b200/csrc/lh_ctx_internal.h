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
    // lh_step_host: p uploads on st_up while the first plane pass runs; the
    // first step's graph waits for ev_p before its first column pass
    cudaStream_t st_up = nullptr;
    cudaEvent_t ev_u = nullptr, ev_p = nullptr;
    cudaGraph_t graph_host = nullptr;
    cudaGraphExec_t gexec_host = nullptr;
    bool have_state = false;
    double *d_spec = nullptr;  // spectra accumulators (lh_diag.cu), allocated on first use
    int spec_count = 0;        // accumulations since the last reset
    double *d_stats = nullptr; // stats accumulators (lh_diag.cu), allocated on first use
    int stats_count = 0;
    lh::StatsScratch stats_scr;  // stats transform scratch and pressure snapshot
    std::string err;
};

// Drop the captured step graphs (a plan change re-captures them on next use).
inline void ctx_drop_graphs(lh_ctx *c)
{
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->gexec_host) cudaGraphExecDestroy(c->gexec_host);
    if (c->graph_host) cudaGraphDestroy(c->graph_host);
    c->gexec = nullptr;
    c->graph = nullptr;
    c->gexec_host = nullptr;
    c->graph_host = nullptr;
}
