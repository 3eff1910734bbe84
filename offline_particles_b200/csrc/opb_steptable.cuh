// The step table of a fused launch (the *_steps entry points): the opb_time
// of every stage of every step.  A device table is read through its pointer;
// a host table travels in the launch's parameters, so the launch needs no
// copy and does not queue behind host-to-device copies issued before it
// (snapshot uploads on another stream share the copy engines).
#pragma once

#include <cuda_runtime.h>

#include <cstring>

#include "opb200.h"
#include "opb_errors.h"

namespace opb {

// Passed as a __grid_constant__ kernel parameter: at() reads the inline
// entries where they are, in the launch's parameter space.
struct StepTable {
    const opb_time *dev;  // device table, or nullptr: the entries are inline
    opb_time inl[OPB_INLINE_TABLE];
    __device__ __forceinline__ opb_time at(int j) const { return dev ? dev[j] : inl[j]; }
};

// Fill `out` for a table of `entries` opb_time at `table`: device memory by pointer, host memory
// (pageable or pinned) by value, each entry's slots checked against `nslots` (the fewest snapshot slots
// of the time-dependent fields; 0: every field static, nothing to check).
inline int make_step_table(const opb_time *table, long long entries, StepTable &out, const char *what,
                           int nslots) {
    out.dev = nullptr;
    if (entries <= 0) return OPB_OK;
    if (!table) return fail(OPB_EINVAL, "%s: step table is NULL", what);
    cudaPointerAttributes attr;
    const cudaError_t e = cudaPointerGetAttributes(&attr, table);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(OPB_ECUDA, "%s: cannot tell where the step table lives: %s", what, cudaGetErrorString(e));
    }
    if (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) {
        out.dev = table;
        return OPB_OK;
    }
    if (entries > OPB_INLINE_TABLE)
        return fail(OPB_EINVAL, "%s: a host step table holds at most %d entries (got %lld); pass a device table",
                    what, OPB_INLINE_TABLE, entries);
    for (long long j = 0; j < entries; ++j)
        if (nslots > 0 && (table[j].prev < 0 || table[j].prev >= nslots || table[j].next < 0 || table[j].next >= nslots))
            return fail(OPB_EINVAL, "%s: step table entry %lld selects slots (%d, %d) of %d", what, j, table[j].prev,
                        table[j].next, nslots);
    memcpy(out.inl, table, (size_t)entries * sizeof(opb_time));
    return OPB_OK;
}

}  // namespace opb
