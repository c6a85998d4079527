// grb_saxpy3.h: the two-phase interface of the row-wise saxpy3 kernels.
//
// saxpy_plan_create runs the symbolic phase once (flop count per row,
// binning, slot capacities, workspace) and may synchronise the host;
// saxpy_plan_exec runs the numeric phase with no allocation and no host
// synchronisation, so it can be captured in a CUDA graph and replayed while
// the operands keep their patterns (values may change between replays).
#pragma once
#include "grb_runtime.h"

namespace grb {

// one shared-memory bin: rows whose flops (+ mask entries) are <= limit go to
// either an expand-sort-compress warp (tpr = 1, cap >= limit product slots)
// or a group of tpr threads (4..32, or 256 for a whole block) with a hash
// table of cap slots (a power of two, at least twice the limit)
struct BinSpec { int64_t limit; int tpr; int cap; };

struct SaxpyConfig {
    int nb = 0;                 // shared-memory bins in use
    BinSpec bin[6];
    int blocks_per_sm = 16;     // persistent grid size of the hash kernels
};

SaxpyConfig saxpy_default_config();
bool saxpy_config_valid(const SaxpyConfig &cfg, size_t zsize);

struct SaxpyPlan;

int saxpy_plan_create(SaxpyPlan **P, const DevCSR *M, bool mask_comp,
                      const DevCSR &A, const DevCSR &B, SemiringCode sr,
                      const SaxpyConfig &cfg, cudaStream_t s);

// capacity (entries) the output arrays of saxpy_plan_exec need
int64_t saxpy_plan_capacity(const SaxpyPlan *P);

// numeric phase: Cp (nrows+1, int32) gets exact row offsets, Cj/Cx the sorted
// rows; nnz = Cp[nrows] (on the device).  Cnnz64 (device, may be null)
// receives nnz as int64.
int saxpy_plan_exec(SaxpyPlan *P, const DevCSR *M, const DevCSR &A,
                    const DevCSR &B, int32_t *Cp, int32_t *Cj, void *Cx,
                    int64_t *Cnnz64, cudaStream_t s);

void saxpy_plan_free(SaxpyPlan *P, cudaStream_t s);

}  // namespace grb
