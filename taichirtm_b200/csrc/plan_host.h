// Host-side plan construction shared by every entry point that builds its own
// tables (rtm_plan_create in rtm_api.cu, rtm_forward_noalloc in noalloc.cu):
// grid validation, the padded row pitch, the sponge profile and the per-row
// source/receiver tables.  One definition, so the entry points cannot drift.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/rtm_b200.h"
#include "step_kernels.cuh"

namespace rtm {

// Grid-level checks of rtm_plan_create; nullptr when the grid is valid, else
// the message.  (The per-shot check, absorbing_frame <= the shot's rows,
// belongs to the shot.)
inline const char *check_grid(const rtm_grid &g) {
    if (g.nx < 3 || g.nz < 3) return "grid must be at least 3x3";
    if (g.nt <= 0) return "nt must be positive";
    if (!(g.fs > 0) || !(g.dx > 0) || !(g.dz > 0)) return "fs, dx, dz must be positive";
    if (g.modes < 1 || g.modes > 3) return "modes must be RTM_PSV, RTM_SH or RTM_BOTH";
    if (g.absorbing_frame < 0 || g.absorbing_frame > g.nz) return "absorbing_frame outside [0, nz]";
    return nullptr;
}

// Floats per padded row.  Lanes touch columns [-vec, nstrips*30*vec + vec);
// with COL_OFF padding columns on the left this fits in ceil(nz/120)*120 + 8
// for every vec (1, 2, 4), so the pitch -- and every caller-visible layout --
// does not depend on the launch shape.  Rounded to 32 floats (128 bytes).
inline int layout_pitch(int nz) { return (((nz + 119) / 120) * 120 + 8 + COL_OFF + 31) / 32 * 32; }

// Sponge profile g(d) = exp(-(a (FW - d))^2), a = 0.0053, d = 0 .. FW-1
// (forward_modeling.py:218-240), evaluated in double and rounded once; at
// least one entry so the device buffer is never empty.
inline std::vector<float> sponge_profile(int fw) {
    std::vector<float> prof(fw > 0 ? fw : 1, 1.0f);
    const double a = 0.0053;
    for (int d = 0; d < fw; ++d) {
        const double diff = (double)(fw - d);
        prof[d] = (float)std::exp((-(a * a) * diff) * diff);
    }
    return prof;
}

// Per-row CSR table of n point entries (i, j) on a window of `rows` rows and
// nz columns: ptr gets rows + 1 offsets appended, ent the (j, base + k) pairs
// row by row, stable in the given order (duplicates accumulate in order).
// Returns -1, or the index of the first entry outside the window (nothing
// is appended then).
inline int append_row_table(int rows, int nz, int n, const int32_t *ij, int base, std::vector<int> &ptr,
                            std::vector<int2> &ent) {
    std::vector<std::vector<int2>> byrow(rows > 0 ? rows : 0);
    for (int k = 0; k < n; ++k) {
        const int i = ij[2 * k], j = ij[2 * k + 1];
        if (i < 0 || i >= rows || j < 0 || j >= nz) return k;
        byrow[i].push_back(make_int2(j, base + k));
    }
    for (int i = 0; i < rows; ++i) {
        ptr.push_back((int)ent.size());
        for (auto &e : byrow[i]) ent.push_back(e);
    }
    ptr.push_back((int)ent.size());
    return -1;
}

// Number of tasks at the end of a work list of n tasks that the tail split
// cuts in two: 8 per SM (a wave of the adjoint kernels, most of one of the
// vec-4 step kernels), at most a quarter of the list.  Measured on the
// 64-shot batched workload: 8 per SM 0.7 % faster than 16, 32 or 48.
inline size_t tail_split_tasks(size_t n, int sms) { return std::min(n / 4, (size_t)(sms > 0 ? sms : 1) * 8); }

// Replace the last `n` tasks {shot, strip word, ia, ib} of `work` that have
// at least 2 rows by their two halves [ia, mid), [mid, ib), in order.
inline void split_tail(std::vector<int4> &work, size_t n) {
    n = std::min(n, work.size());
    const size_t head = work.size() - n;
    std::vector<int4> tail;
    tail.reserve(2 * n);
    for (size_t t = head; t < work.size(); ++t) {
        const int4 w = work[t];
        if (w.w - w.z >= 2) {
            const int mid = w.z + (w.w - w.z + 1) / 2;
            tail.push_back(make_int4(w.x, w.y, w.z, mid));
            tail.push_back(make_int4(w.x, w.y, mid, w.w));
        } else {
            tail.push_back(w);
        }
    }
    work.resize(head);
    work.insert(work.end(), tail.begin(), tail.end());
}

}  // namespace rtm
