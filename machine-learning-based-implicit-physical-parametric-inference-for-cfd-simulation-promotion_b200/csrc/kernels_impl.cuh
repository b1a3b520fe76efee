// kernels_impl.cuh -- instantiates and launches the step kernels of one
// storage type, dispatching operator and scene at run time.
#pragma once

#include "launch.h"

namespace ippi {

template <int S, int CO, int SC>
static cudaError_t launch_tpl(const LaunchSet& L)
{
    const bool side = L.nprep > 0;
    if (side) {
        cudaEventRecord(L.fork, L.stream);
        cudaStreamWaitEvent(L.side, L.fork, 0);
        if (L.events) cudaEventRecord(L.events[2], L.side);
        prep_kernel<S, SC><<<(L.nprep + 255) / 256, 256, 0, L.side>>>(L.step, L.prep, L.nprep);
        if (L.band) band_kernel<S, CO><<<L.band_blocks, kBandThreads, 0, L.side>>>(L.band_args);
        if (L.ib) {
            if (L.ib_nst == 16)
                ib_kernel<S, CO, 16><<<L.ib_blocks, kIbThreads, L.ib_smem, L.side>>>(L.ib_args);
            else
                ib_kernel<S, CO, 4><<<L.ib_blocks, kIbThreads, L.ib_smem, L.side>>>(L.ib_args);
        }
        if (L.events) cudaEventRecord(L.events[3], L.side);
        cudaEventRecord(L.join, L.side);
    }
    if (L.events) cudaEventRecord(L.events[0], L.stream);
    step_kernel<S, CO, SC><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
    if (L.events) cudaEventRecord(L.events[1], L.stream);
    if (side) cudaStreamWaitEvent(L.stream, L.join, 0);
    return cudaGetLastError();
}

template <int S>
static cudaError_t launch_store(const LaunchSet& L)
{
    if (L.scene == SC_REF) {
        switch (L.coll) {
        case CO_MRT: return launch_tpl<S, CO_MRT, SC_REF>(L);
        case CO_RR: return launch_tpl<S, CO_RR, SC_REF>(L);
        default: return launch_tpl<S, CO_BGK, SC_REF>(L);
        }
    }
    switch (L.coll) {
    case CO_MRT: return launch_tpl<S, CO_MRT, SC_CHANNEL>(L);
    case CO_RR: return launch_tpl<S, CO_RR, SC_CHANNEL>(L);
    default: return launch_tpl<S, CO_BGK, SC_CHANNEL>(L);
    }
}

template <int S>
static cudaError_t prepare_store(size_t smem)
{
    const int v = (int)smem;
    cudaError_t e = cudaSuccess;
#define IPPI_SMEM(CO, N)                                                                     \
    if (e == cudaSuccess)                                                                    \
        e = cudaFuncSetAttribute(ib_kernel<S, CO, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    IPPI_SMEM(CO_BGK, 4) IPPI_SMEM(CO_BGK, 16) IPPI_SMEM(CO_MRT, 4) IPPI_SMEM(CO_MRT, 16)
    IPPI_SMEM(CO_RR, 4) IPPI_SMEM(CO_RR, 16)
#undef IPPI_SMEM
    return e;
}

}  // namespace ippi
