"""How a fused Euler stage splits into launches over fewer staged inputs
(split_by_inputs, x3div_b200/csrc/stage_split.h), checked on the CPU: a small
C++ program built with g++ against the library's headers runs the split on
hand-made stage programs (no GPU, no kernel launch)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "x3div_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"

HARNESS = r"""
#include <cstdio>
#include "stage_split.h"
using namespace x3d;
static float buf[64];
static const float *IN(int i) { return buf + i; }       // distinct staged inputs
static void *OUT(int i) { return buf + 32 + i; }         // distinct outputs
static StageOp<float> op(int a, int b, int m, int acc, int flush, void *out, const void *base = nullptr)
{
    StageOp<float> o;
    std::memset(&o, 0, sizeof(o));
    o.src_a = (short)a; o.src_b = (short)b; o.mul_tile = (short)m;
    o.accumulate = (short)acc; o.flush = (short)flush; o.out = out; o.base = base;
    return o;
}
static void show(const char *name, const StageProgram<float> &p)
{
    StageProgram<float> part[kMaxStageOps];
    const int n = split_by_inputs<float>(p, part);
    std::printf("%s %d", name, n);
    for (int q = 0; q < n && n > 1; ++q) {
        std::printf(" |");
        for (int t = 0; t < part[q].ntiles; ++t) std::printf(" in%d", (int)(part[q].in[t] - buf));
        for (int k = 0; k < part[q].nops; ++k) {
            const StageOp<float> &o = part[q].ops[k];
            if (o.out)
                std::printf(" op(%d,%d,%d,out%d)", o.src_a, o.src_b, o.mul_tile,
                            (int)((float *)o.out - buf) - 32);
            else
                std::printf(" op(%d,%d,%d,out-)", o.src_a, o.src_b, o.mul_tile);
        }
    }
    std::printf("\n");
}
int main()
{
    StageProgram<float> p;
    // divergence x: three independent one-operator chains, one per input
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 3; p.in[0] = IN(0); p.in[1] = IN(1); p.in[2] = IN(2); p.nops = 3;
    p.ops[0] = op(0, -1, -1, 0, 1, OUT(0)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1));
    p.ops[2] = op(2, -1, -1, 0, 1, OUT(2));
    show("three", p);
    // momentum: every chain reads u_d (tile 0)
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 3; p.in[0] = IN(0); p.in[1] = IN(1); p.in[2] = IN(2); p.nops = 6;
    for (int c = 0; c < 3; ++c) {
        p.ops[2 * c] = op(c, -1, 0, 0, 0, nullptr);
        p.ops[2 * c + 1] = op(0, c, -1, 1, 1, OUT(c));
    }
    show("shared", p);
    // divergence y: one chain over tiles 0 and 1 (summed), one over tile 2
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 3; p.in[0] = IN(0); p.in[1] = IN(1); p.in[2] = IN(2); p.nops = 3;
    p.ops[0] = op(0, -1, -1, 0, 0, nullptr); p.ops[1] = op(1, -1, -1, 1, 1, OUT(0));
    p.ops[2] = op(2, -1, -1, 0, 1, OUT(1));
    show("pair", p);
    // chains on {0}, {1} and then {0, 1}: the third joins the first two
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 2; p.in[0] = IN(0); p.in[1] = IN(1); p.nops = 3;
    p.ops[0] = op(0, -1, -1, 0, 1, OUT(0)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1));
    p.ops[2] = op(0, 1, -1, 0, 1, OUT(2));
    show("merge", p);
    // chains on {0}, {1}, {2}, {1, 2}: two parts, {0} and {1, 2}
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 3; p.in[0] = IN(0); p.in[1] = IN(1); p.in[2] = IN(2); p.nops = 4;
    p.ops[0] = op(0, -1, -1, 0, 1, OUT(0)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1));
    p.ops[2] = op(2, -1, -1, 0, 1, OUT(2)); p.ops[3] = op(1, 2, -1, 0, 1, OUT(3));
    show("late", p);
    // one part writes the array another part stages: no split
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 2; p.in[0] = IN(0); p.in[1] = IN(1); p.nops = 2;
    p.ops[0] = op(0, -1, -1, 0, 1, (void *)IN(1)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1));
    show("hazard_in", p);
    // one part writes the array another part reads as its base: no split
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 2; p.in[0] = IN(0); p.in[1] = IN(1); p.nops = 2;
    p.ops[0] = op(0, -1, -1, 0, 1, OUT(0)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1), OUT(0));
    show("hazard_base", p);
    // in-place flushes (base = out) within one part are fine
    std::memset(&p, 0, sizeof(p));
    p.ntiles = 2; p.in[0] = IN(0); p.in[1] = IN(1); p.nops = 2;
    p.ops[0] = op(0, -1, -1, 0, 1, OUT(0), OUT(0)); p.ops[1] = op(1, -1, -1, 0, 1, OUT(1), OUT(1));
    show("inplace", p);
    return 0;
}
"""


@pytest.fixture(scope="module")
def results(tmp_path_factory):
    if not shutil.which("g++") or not os.path.isdir(CUDA_INC):
        pytest.skip("needs g++ and the CUDA headers")
    d = tmp_path_factory.mktemp("split")
    src, exe = d / "split.cpp", d / "split"
    src.write_text(HARNESS)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, "-I", CUDA_INC, str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {line.split()[0]: line.split(" ", 1)[1] for line in out.strip().splitlines()}


def test_independent_chains_split_one_launch_per_input(results):
    assert results["three"] == ("3 | in0 op(0,-1,-1,out0) | in1 op(0,-1,-1,out1) | in2 op(0,-1,-1,out2)")


def test_chains_sharing_an_input_stay_together(results):
    assert results["shared"] == "1"
    assert results["merge"] == "1"


def test_inputs_are_renumbered_within_each_part(results):
    assert results["pair"] == "2 | in0 in1 op(0,-1,-1,out-) op(1,-1,-1,out0) | in2 op(0,-1,-1,out1)"
    assert results["late"] == ("2 | in0 op(0,-1,-1,out0) | in1 in2 op(0,-1,-1,out1) op(1,-1,-1,out2) "
                               "op(0,1,-1,out3)")


def test_no_split_where_a_part_writes_what_another_reads(results):
    assert results["hazard_in"] == "1"
    assert results["hazard_base"] == "1"
    assert results["inplace"].startswith("2 ")
