"""Checkpoint files in the reference's formats (print2D, printHeating) and the
binary checkpoint/restart.  The golden files are the reference's own output
of the final state of two golden cases (tests/golden/make_golden.py)."""
import os
import tempfile

import numpy as np
import pytest

import common
import torch_b200
from torch_b200 import snapshot

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def assert_tables_close(path_got, path_ref, rtol=1e-9):
    """Relative agreement per value, with an absolute floor of rtol times the
    column's largest magnitude (values like an HII fraction of 1e-290 carry no
    digits that two libm implementations agree on)."""
    t1, n1, a = snapshot.read_table(path_got)
    t2, n2, b = snapshot.read_table(path_ref)
    assert n1 == n2 and a.shape == b.shape
    assert abs(t1 - t2) <= rtol * abs(t2)
    both_nan = np.isnan(a) & np.isnan(b)
    diff = np.abs(a - b)
    scale = np.nanmax(np.abs(b), axis=0, keepdims=True)
    ok = both_nan | (diff <= rtol * np.maximum(np.abs(a), np.abs(b)) + rtol * scale + 1e-300)
    assert ok.all(), (np.argwhere(~ok)[:5], a[~ok][:5], b[~ok][:5])


@pytest.mark.parametrize("name", ["blister_small", "hii3d_small"])
def test_data2d_writer_matches_reference_output(name):
    """The print2D restatement, fed the reference's own final primitives,
    reproduces the reference's file (CPU only)."""
    tp, ic, steps, ref = common.load_golden(name)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "data2D.txt.gz")
        snapshot.write_data2d(out, tp, ic.ncells, ref["Q"], float(ref["time"]))
        assert_tables_close(out, os.path.join(GOLD, f"ckpt_{name}_data2D.txt.gz"), rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["blister_small", "hii3d_small"])
def test_checkpoint_files_match_reference(name):
    """A GPU run with the heating diagnostics on writes the checkpoint files
    the reference writes for the same run (values to 1e-9: the files carry
    11 significant digits)."""
    tp, ic, steps, ref = common.load_golden(name)
    sim = torch_b200.Torch(tp, ic)
    sim.heating_enable(True)
    sim.run_steps(steps)
    with tempfile.TemporaryDirectory() as d:
        snapshot.write_checkpoint(d, sim, tp, ic.ncells)
        for kind in ("data2D", "heating"):
            assert_tables_close(os.path.join(d, f"{kind}_final.txt.gz"),
                                os.path.join(GOLD, f"ckpt_{name}_{kind}.txt.gz"))
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", ["fp64", "fp32"])
def test_checkpoint_restart_is_bitwise(form):
    """Save after 6 steps, go on 6 steps; a fresh context restored from the
    save and stepped 6 times ends bit-for-bit at the same state."""
    from torch_b200 import workloads
    tp, ic = workloads.hii_region(n=16, seed=3)
    prec = torch_b200.PRECISION_FP64 if form == "fp64" else torch_b200.PRECISION_FP32
    a = torch_b200.Torch(tp, ic, precision=prec)
    a.run_steps(6)
    blob = a.checkpoint()
    a.run_steps(6)
    sa = a.state()
    a.close()
    b = torch_b200.Torch(tp, ic, precision=prec)
    b.restore(blob)
    b.run_steps(6)
    sb = b.state()
    b.close()
    for k in ("U", "Q", "R", "T"):
        assert np.array_equal(getattr(sa, k), getattr(sb, k)), k
    assert sa.time == sb.time


@pytest.mark.gpu
def test_checkpoint_moves_between_fp64_and_fp32_forms():
    """A radiation-hydro run switches precision mid-run: an FP64-form
    checkpoint restored into an FP32-form context continues within the FP32
    form's error of the FP64 run, and that context's checkpoint restored into
    an FP64-form context holds the same state arrays bit for bit."""
    from torch_b200 import workloads
    tp, ic = workloads.hii_region(n=16, seed=3)
    a = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP64)
    a.run_steps(6)
    blob = a.checkpoint()
    a.run_steps(6)
    sa = a.state()
    a.close()
    b = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP32)
    b.restore(blob)
    b.run_steps(6)
    sb = b.state()
    blob_b = b.checkpoint()
    b.close()
    for i in (0, 1, 2):
        assert common.rel_l1(sb.U[i], sa.U[i]) <= 1e-5, i
    assert abs(sb.time - sa.time) <= 1e-6 * sa.time  # the forms' CFL steps differ by rounding
    c = torch_b200.Torch(tp, ic, precision=torch_b200.PRECISION_FP64)
    c.restore(blob_b)
    sc = c.state()
    c.close()
    for k in ("U", "R", "T"):
        assert np.array_equal(getattr(sb, k), getattr(sc, k)), k


@pytest.mark.gpu
def test_checkpoint_rejects_other_grid():
    from torch_b200 import workloads
    tp, ic = workloads.hii_region(n=16, seed=3)
    a = torch_b200.Torch(tp, ic)
    blob = a.checkpoint()
    a.close()
    tp2, ic2 = workloads.hii_region(n=12, seed=3)
    b = torch_b200.Torch(tp2, ic2)
    with pytest.raises(torch_b200.TrgError):
        b.restore(blob)
    b.close()
