// ORACLE / baseline infrastructure — not product code.
//
// Host launcher for the reference's own GPU kernels wfkerneld / wfkernelf
// (idi/simulation/sim.cu:141-149), compiled from the reference tree (the
// file named by REF_SIM_CU; see oracle/Makefile) for sm_100a with the
// settings "nf" (-Dusenf), no 1/r (-Dnodist), no detector rotation
// (-Dnodetrot) and --use_fast_math, and launched with the reference's
// 16x16 thread blocks (idi/simulation/cuda.py:76-79).  Used only to time the
// reference GPU path next to this project's kernels.
#define usenf 1
#define nodist 1
#define nodetrot 1
#include REF_SIM_CU

extern "C" int ref_wf_launch(int single, void *ret, const void *atoms, float detx, float dety, float detz,
                             float pixelsize, float k, int maxx, int maxy, int natoms, void *stream) {
    dim3 block(16, 16, 1);
    dim3 grid((maxx + 15) / 16, (maxy + 15) / 16);
    if (single)
        wfkernelf<<<grid, block, 0, (cudaStream_t)stream>>>((float2 *)ret, (const float4 *)atoms, nullptr, detx, dety,
                                                             detz, pixelsize, k, maxx, maxy, natoms);
    else
        wfkerneld<<<grid, block, 0, (cudaStream_t)stream>>>((double2 *)ret, (const double4 *)atoms, nullptr, detx,
                                                              dety, detz, pixelsize, k, maxx, maxy, natoms);
    return (int)cudaGetLastError();
}
