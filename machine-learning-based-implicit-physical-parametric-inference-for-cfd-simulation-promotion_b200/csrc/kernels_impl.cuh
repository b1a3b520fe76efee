// kernels_impl.cuh -- instantiates and launches the step kernels of one
// storage type, dispatching operator and scene at run time.
#pragma once

#include "launch.h"

namespace ippi {

// Side-stream kernels carry an explicit launch priority, so the priority
// survives stream capture into the step graphs and their blocks take the
// first free slots while the bulk kernel fills the GPU.
template <typename... KArgs, typename... Args>
static void launch_prio(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t st,
                        int prio, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = prio;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int S, int SC, int CO, bool LRN, int XT = 0>
static void launch_ib(const LaunchSet& L, cudaStream_t st)
{
    // the whole IB sub-step: one cluster of kIbCtas CTAs
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kIbCtas);
    cfg.blockDim = dim3(kIbThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = L.side_prio;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = kIbCtas;
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    if (L.ib_nst == 16)
        cudaLaunchKernelEx(&cfg, ib_fused<S, SC, CO, LRN, 16, XT>, L.ib_args, L.ib_passes);
    else
        cudaLaunchKernelEx(&cfg, ib_fused<S, SC, CO, LRN, 4, XT>, L.ib_args, L.ib_passes);
}

// the bulk kernel of a normal step (with or without the running means)
template <int S, int CO, int SC, bool LRN, int XT>
static void launch_bulk(const LaunchSet& L)
{
    if (L.avg_on)
        step_fast<S, CO, SC, LRN, XT, 1><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
    else
        step_fast<S, CO, SC, LRN, XT, 0><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
}

// a normal step with markers as one launch: the IB blocks first, then the
// bulk row segments (step_ib_fused)
template <int S, int CO, int SC, bool LRN, int XT>
static void launch_merged(const LaunchSet& L)
{
    const unsigned nblk = (unsigned)L.ib_args.nib + L.grid.x * L.grid.y;
    IbArgs ia = L.ib_args;
    ia.s = L.step;
    if (L.ib_nst == 16) {
        if (L.avg_on)
            step_ib_fused<S, SC, CO, LRN, 16, XT, 1><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
        else
            step_ib_fused<S, SC, CO, LRN, 16, XT, 0><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
    } else {
        if (L.avg_on)
            step_ib_fused<S, SC, CO, LRN, 4, XT, 1><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
        else
            step_ib_fused<S, SC, CO, LRN, 4, XT, 0><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
    }
}

// the boundary nets' kernel (dynamic shared memory: two weight buffers and
// the activations, allowed once per device by band_setup); `pdl`: launched as
// the programmatic dependent of the kernel before it on the stream
template <int S, int CO>
static void launch_band(const LaunchSet& L, cudaStream_t st, bool pdl)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.band_blocks);
    cfg.blockDim = dim3(kBandThreads);
    cfg.dynamicSmemBytes = BandShapeOf<S>::SmemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = L.side_prio;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 2 : 1;
    cudaLaunchKernelEx(&cfg, band_kernel<S, CO>, L.band_args);
}

// A normal step with boundary nets (no markers), in one stream: prep_kernel,
// then band_kernel as its programmatic dependent, then the bulk kernel as
// band_kernel's.  Each primary lets its dependent launch from its first
// instruction, so the band blocks are resident (waiting for prep's moments)
// before the bulk row segments take the rest of the GPU, and the nets run
// beside the bulk step instead of after it.  The bulk grid's last block waits
// for band_kernel's completion, so the step ends after all three.
template <int S, int CO, int SC>
static void launch_band_step(const LaunchSet& L)
{
    launch_prio(prep_kernel<S, SC>, (L.nprep + 255) / 256, 256, L.stream, L.side_prio, L.step, L.prep, L.nprep);
    launch_band<S, CO>(L, L.stream, true);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = L.grid;
    cfg.blockDim = dim3(kBlockX);
    cfg.stream = L.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (L.avg_on)
        cudaLaunchKernelEx(&cfg, step_fast<S, CO, SC, false, 0, 1>, L.step);
    else
        cudaLaunchKernelEx(&cfg, step_fast<S, CO, SC, false, 0, 0>, L.step);
}

template <int S, int CO, int SC, bool LRN, int XT = 0>
static cudaError_t launch_tpl(const LaunchSet& L)
{
    // Closures that read neighbour velocities (WALE, coherent structure):
    // the post-stream velocities of all nodes first, then the IB kernel
    // (which overwrites its nodes' with the corrected ones), then the bulk
    // kernel, in stream order; the local models (tau field, wall-damped Cs)
    // in timed launches.  Channel scene only: no boundary-net work.
    if (XT && (L.step.les == 3 || L.step.les == 6) && L.step.mode == MODE_STEP && L.ib && !L.events) {
        // the tau field and the wall-damped closure are local: one launch
        // with the IB blocks, as the normal step below
        launch_merged<S, CO, SC, LRN, XT>(L);
        return cudaGetLastError();
    }
    if (XT && (L.step.les == 4 || L.step.les == 5) && L.step.mode == MODE_STEP && L.ib && !L.events) {
        // WALE / coherent model with markers: two launches, the IB force
        // phases beside the velocity pass, then the forced collisions beside
        // the bulk row segments
        IbArgs ia = L.ib_args;
        ia.s = L.step;
        const unsigned nblk = (unsigned)kIbCtas + L.grid.x * L.grid.y;
        if (L.ib_nst == 16)
            mac_ib_fused<S, SC, 16><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
        else
            mac_ib_fused<S, SC, 4><<<nblk, kBlockX, 0, L.stream>>>(ia, L.ib_passes);
        if (L.avg_on)
            collide_ib_fused<S, SC, CO, LRN, 1><<<nblk, kBlockX, 0, L.stream>>>(ia);
        else
            collide_ib_fused<S, SC, CO, LRN, 0><<<nblk, kBlockX, 0, L.stream>>>(ia);
        return cudaGetLastError();
    }
    if (XT) {
        // timed launches: events 2-3 around the velocity pass and the IB
        // kernel, 0-1 around the bulk kernel
        if (L.events) cudaEventRecord(L.events[2], L.stream);
        if (L.step.les == 4 || L.step.les == 5) mac_kernel<S, SC><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
        if (L.ib) launch_ib<S, SC, CO, LRN, XT>(L, L.stream);
        if (L.events) {
            cudaEventRecord(L.events[3], L.stream);
            cudaEventRecord(L.events[0], L.stream);
        }
        if (L.step.mode == MODE_STEP)
            launch_bulk<S, CO, SC, LRN, XT>(L);
        else
            step_kernel<S, CO, SC, LRN, XT><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
        if (L.events) cudaEventRecord(L.events[1], L.stream);
        return cudaGetLastError();
    }
    // Normal steps with markers and no boundary nets: one launch, IB blocks
    // and bulk row segments.  Timed launches (events) keep the side-stream
    // form below, so the bulk kernel's own duration can be measured.
    if (L.step.mode == MODE_STEP && L.ib && !L.band && L.nprep == 0 && !L.events) {
        launch_merged<S, CO, SC, LRN, 0>(L);
        return cudaGetLastError();
    }
    if (!LRN && !XT && L.step.mode == MODE_STEP && L.band && L.nprep > 0 && !L.ib && !L.events) {
        launch_band_step<S, CO, SC>(L);
        return cudaGetLastError();
    }
    const bool side = L.nprep > 0 || L.band || L.ib;
    if (side) {
        cudaEventRecord(L.fork, L.stream);
        cudaStreamWaitEvent(L.side, L.fork, 0);
        if (L.events) cudaEventRecord(L.events[2], L.side);
        if (L.nprep > 0)
            launch_prio(prep_kernel<S, SC>, (L.nprep + 255) / 256, 256, L.side, L.side_prio, L.step,
                        L.prep, L.nprep);
        if (L.band) launch_band<S, CO>(L, L.side, false);
        if (L.ib) launch_ib<S, SC, CO, LRN>(L, L.side);
        if (L.events) cudaEventRecord(L.events[3], L.side);
        cudaEventRecord(L.join, L.side);
    }
    if (L.events) cudaEventRecord(L.events[0], L.stream);
    if (L.step.mode == MODE_STEP)
        launch_bulk<S, CO, SC, LRN, 0>(L);
    else
        step_kernel<S, CO, SC, LRN><<<L.grid, kBlockX, 0, L.stream>>>(L.step);
    if (L.events) cudaEventRecord(L.events[1], L.stream);
    if (side) cudaStreamWaitEvent(L.stream, L.join, 0);
    return cudaGetLastError();
}

// the boundary-net kernels' dynamic shared memory above the 48 KB default
// (current device; outside any stream capture)
template <int S>
static cudaError_t band_setup()
{
    for (cudaError_t e : {cudaFuncSetAttribute(band_kernel<S, CO_BGK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)BandShapeOf<S>::SmemBytes),
                          cudaFuncSetAttribute(band_kernel<S, CO_MRT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)BandShapeOf<S>::SmemBytes),
                          cudaFuncSetAttribute(band_kernel<S, CO_RR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)BandShapeOf<S>::SmemBytes)})
        if (e != cudaSuccess) return e;
    return cudaSuccess;
}

template <int S>
static cudaError_t launch_store(const LaunchSet& L)
{
    if (L.scene == SC_REF) {
        switch (L.coll) {
        case CO_MRT: return launch_tpl<S, CO_MRT, SC_REF, false>(L);
        case CO_RR: return launch_tpl<S, CO_RR, SC_REF, false>(L);
        default: return launch_tpl<S, CO_BGK, SC_REF, false>(L);
        }
    }
    // the tau field (3) and the closures 4..6 are built for the channel scene
    if (L.step.les >= 3) {
        switch (L.coll) {
        case CO_MRT: return launch_tpl<S, CO_MRT, SC_CHANNEL, false, 1>(L);
        case CO_RR: return launch_tpl<S, CO_RR, SC_CHANNEL, false, 1>(L);
        default: return launch_tpl<S, CO_BGK, SC_CHANNEL, false, 1>(L);
        }
    }
    // the learned relaxation time (les == 2) is built for the channel scene
    if (L.step.les == 2) {
        switch (L.coll) {
        case CO_MRT: return launch_tpl<S, CO_MRT, SC_CHANNEL, true>(L);
        case CO_RR: return launch_tpl<S, CO_RR, SC_CHANNEL, true>(L);
        default: return launch_tpl<S, CO_BGK, SC_CHANNEL, true>(L);
        }
    }
    switch (L.coll) {
    case CO_MRT: return launch_tpl<S, CO_MRT, SC_CHANNEL, false>(L);
    case CO_RR: return launch_tpl<S, CO_RR, SC_CHANNEL, false>(L);
    default: return launch_tpl<S, CO_BGK, SC_CHANNEL, false>(L);
    }
}

}  // namespace ippi
