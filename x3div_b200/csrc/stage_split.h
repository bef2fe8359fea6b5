// Splitting a stage program into launches over fewer staged inputs
// (used by stages.cpp; host code only).
#pragma once

#include <cstring>

#include "linesolve_chunk.h"

namespace x3d {

// A program's operators in launches over fewer staged inputs: the operators
// from an accumulator's start to its flush stay together, and such chains
// that share no staged input go to different launches, which stage fewer
// bytes per line and so fit more CTAs on an SM.  Returns the number of
// parts (1: the program does not split, or a part would write an array
// another part reads).
template <typename T>
inline int split_by_inputs(const StageProgram<T> &p, StageProgram<T> (&part)[kMaxStageOps])
{
    int chain[kMaxStageOps], nchains = 0;
    unsigned uses[kMaxStageOps] = {};  // bit t: chain reads staged input t
    for (int k = 0; k < p.nops; ++k) {
        const StageOp<T> &o = p.ops[k];
        if (k == 0 || !o.accumulate) ++nchains;
        chain[k] = nchains - 1;
        unsigned &u = uses[nchains - 1];
        for (const int t : {(int)o.src_a, (int)o.src_b, (int)o.mul_tile})
            if (t >= 0) u |= 1u << t;
    }
    // chains that share an input go together (groups in order of first use)
    int group[kMaxStageOps], ngroups = 0;
    unsigned gin[kMaxStageOps] = {};
    for (int c = 0; c < nchains; ++c) {
        int g = -1;
        for (int h = 0; h < ngroups && g < 0; ++h)
            if (gin[h] & uses[c]) g = h;
        if (g < 0) g = ngroups++;
        gin[g] |= uses[c];
        group[c] = g;
        // a chain joining a group may connect it to a later group: merge them
        for (int h = g + 1; h < ngroups; ++h)
            if (gin[h] & gin[g]) {
                gin[g] |= gin[h];
                for (int e = 0; e < c; ++e)
                    if (group[e] == h) group[e] = g;
                gin[h] = 0;
            }
    }
    // renumber the groups that are left, in order of first use
    int ren[kMaxStageOps], nparts = 0;
    for (int h = 0; h < ngroups; ++h) ren[h] = -1;
    for (int c = 0; c < nchains; ++c)
        if (ren[group[c]] < 0) ren[group[c]] = nparts++;
    if (nparts < 2) return 1;
    // no part may write an array that another part reads
    for (int a = 0; a < p.nops; ++a)
        for (int b = 0; b < p.nops; ++b) {
            const StageOp<T> &w = p.ops[a], &r = p.ops[b];
            if (ren[group[chain[a]]] == ren[group[chain[b]]]) continue;
            for (const void *out : {(const void *)w.out, (const void *)w.out2}) {
                if (!out) continue;
                if (out == r.base || out == r.base2) return 1;
                for (const int t : {(int)r.src_a, (int)r.src_b, (int)r.mul_tile})
                    if (t >= 0 && out == p.in[t]) return 1;
            }
        }
    for (int q = 0; q < nparts; ++q) {
        StageProgram<T> &s = part[q];
        std::memset(&s, 0, sizeof(s));
        s.in_f64 = p.in_f64;
        int map[kMaxStageTiles];
        for (int t = 0; t < p.ntiles; ++t) map[t] = -1;
        for (int k = 0; k < p.nops; ++k) {
            if (ren[group[chain[k]]] != q) continue;
            StageOp<T> o = p.ops[k];
            for (short *t : {&o.src_a, &o.src_b, &o.mul_tile})
                if (*t >= 0) {
                    if (map[*t] < 0) {
                        map[*t] = s.ntiles;
                        s.in[s.ntiles++] = p.in[*t];
                    }
                    *t = (short)map[*t];
                }
            s.ops[s.nops++] = o;
        }
    }
    return nparts;
}

}  // namespace x3d
