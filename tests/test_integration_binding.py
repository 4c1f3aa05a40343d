"""The reference-side C++ binding shown in INTEGRATION.md (class TorchGPU)
compiles, exactly as written there, against the reference's own headers and
include/torch_b200.h, and links with libtorch_b200.so and the reference
objects it uses (Constants' enum parsers).  Needs the reference tree and its
build (oracle/_ref), i.e. this build container; skipped elsewhere.  The
linked program is run without arguments, which makes no CUDA call."""
import os
import re
import shutil
import subprocess
import tempfile

import pytest

import common
import oracle
import torch_b200

MAIN = r"""
#include "TorchGPU.hpp"
#include <cstdio>

// A caller of the binding: constructed only when asked to (never in the test).
int main(int argc, char** argv) {
    if (argc > 1) {
        TorchParameters p;
        std::vector<double> den(1, 1e-20), pre(1, 1e-12), hii(1, 0), v(1, 0);
        TorchGPU gpu(p, den, pre, hii, v, v, v);
        double dt = gpu.fullStep(1.0);
        std::vector<double> U, Q;
        gpu.state(U, Q);
        std::printf("%g %zu\n", dt, U.size());
    }
    std::printf("binding linked\n");
    return 0;
}
"""


def binding_source():
    text = open(os.path.join(common.ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    src = [b for b in blocks if "class TorchGPU" in b]
    assert len(src) == 1, "INTEGRATION.md must hold exactly one TorchGPU block"
    return src[0]


def test_torchgpu_binding_compiles_and_links():
    ref = oracle.REF_TREE
    objdir = os.path.join(common.ROOT, "oracle", "_ref", "obj")
    if not os.path.isdir(os.path.join(ref, "src")) or not os.path.isdir(objdir):
        pytest.skip("reference tree or its build (oracle/_ref) unavailable")
    lib = torch_b200.library_path()
    assert os.path.exists(lib), "libtorch_b200.so missing: run __graft_entry__.build()"
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "TorchGPU.hpp"), "w") as f:
            f.write("#pragma once\n" + binding_source())
        with open(os.path.join(d, "main.cpp"), "w") as f:
            f.write(MAIN)
        shim = os.path.join(common.ROOT, "oracle", "ref", "shim")
        objs = [os.path.join(objdir, "Torch", n) for n in ("Constants.o", "Converter.o")]
        cmd = ["g++", "-std=c++11", "-w", "-I" + d, "-I" + shim, "-I" + os.path.join(ref, "src"),
               "-I" + os.path.join(ref, "lib"), "-I" + os.path.join(common.ROOT, "include"),
               os.path.join(d, "main.cpp")] + objs + \
              ["-L" + os.path.dirname(lib), "-ltorch_b200", "-Wl,-rpath," + os.path.dirname(lib),
               "-o", os.path.join(d, "binding")]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-3000:]
        out = subprocess.run([os.path.join(d, "binding")], capture_output=True, text=True, timeout=60)
        assert out.returncode == 0 and "binding linked" in out.stdout, out.stderr


def test_slab_hook_example_compiles():
    """The NCCL exchange hook of INTEGRATION.md's decomposed-run example,
    compiled against the library header and the system NCCL header, with
    the calls it makes to register itself and the sweep buffers."""
    if not os.path.exists("/usr/include/nccl.h"):
        pytest.skip("no NCCL header")
    text = open(os.path.join(common.ROOT, "INTEGRATION.md")).read()
    blocks = [b for b in re.findall(r"```cpp\n(.*?)```", text, flags=re.S) if "trg_exchange_fn" in b]
    assert len(blocks) == 1
    body = blocks[0].replace("trg_slab_exchange(ctx, exchange, &comm, send, recv, dt);",
                             "void reg(trg_ctx* ctx, SlabComm& comm, void* send, void* recv, void* dt) {\n"
                             "    trg_slab_exchange(ctx, exchange, &comm, send, recv, dt);\n}")
    body = body.replace("trg_slab_sweep_exchange(ctx, sw_send, sw_recv);",
                        "void reg_sweeps(trg_ctx* ctx, void* sw_send, void* sw_recv) {\n"
                        "    trg_slab_sweep_exchange(ctx, sw_send, sw_recv);\n}")
    src = "#include <cuda_runtime.h>\n#include <nccl.h>\n#include \"torch_b200.h\"\n" + body
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "hook.cpp"), "w") as f:
            f.write(src)
        cuda_inc = os.path.join(os.path.dirname(os.path.dirname(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")),
                                "include")
        cmd = ["g++", "-std=c++11", "-c", "-I" + os.path.join(common.ROOT, "include"), "-I" + cuda_inc,
               os.path.join(d, "hook.cpp"), "-o", os.path.join(d, "hook.o")]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr[-3000:]
