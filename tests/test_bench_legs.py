"""Host logic of two bench legs with the library and the CUDA events replaced by fakes (no GPU): the general-operator
leg builds edc_setup's o for every group and times both operator forms; the adjoint leg reports the differences of the
allocating and checkpointed gradients; a leg that raises is reported in the line."""
import numpy as np
import pytest
import torch

import asr_b200 as A
import bench


class _Event:
    def __init__(self, **kw):
        pass

    def record(self, stream=None):
        pass

    def elapsed_time(self, other):
        return 10.0


class _Ctx:
    def __init__(self):
        self.held = []

    def hold_workspace(self, on):
        self.held.append(bool(on))

    def profile(self, on):
        pass

    def kernel_stats(self, kind):
        return {"ms": 2.0, "launches": 4, "bytes": 1.0, "flops": 1.0}


class _Op:
    def __init__(self):
        self.ctx = _Ctx()


@pytest.fixture
def fake_cuda(monkeypatch):
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda: None)


@pytest.fixture(scope="module")
def workload():
    return bench.workload()


def test_general_leg_runs_both_operator_forms(fake_cuda, workload):
    _, _, groups, z_all = workload
    seen = []

    class Lib:
        ChainSpec = A.ChainSpec

        @staticmethod
        def chains_run(op, specs, z, mode, depth_tol, tail, precision):
            seen.append((any(np.any(np.asarray(s.o) != 0) for s in specs), len(z), precision))
            return {"g": np.zeros((len(z), len(specs)), complex)}

    class Args:
        nz_slice = 192

    op = _Op()
    out = bench.general_leg(Args, Lib, op, groups, z_all, None)
    assert [s[0] for s in seen] == [True, True, False, False]   # o from edc_setup, then o = 0; warm-up and timed each
    assert [s[1] for s in seen] == [32, 192, 32, 192] and {s[2] for s in seen} == {"fp64"}
    steps = sum(g["nlev"] for g in groups) * 192
    assert out["o_edc_setup"]["chain_steps_per_s"] == pytest.approx(steps / 0.01)
    assert out["o_zero_over_o_edc_setup"] == pytest.approx(1.0)
    assert op.ctx.held == [True, False]


def test_adjoint_leg_reports_mode_differences(fake_cuda, workload):
    _, _, groups, z_all = workload

    class Lib:
        @staticmethod
        def chains_adjoint(op, specs, z, w, tail, precision, project, stride=0):
            return None, np.ones((len(specs), 3, 3, 9), complex) * (1.0 + 1e-15 * stride)

        @staticmethod
        def chains_run(op, specs, z, mode, depth_tol, tail, precision):
            return {"g": np.zeros((len(z), len(specs)), complex)}

    class Args:
        adj_groups, adj_depth, adj_energies = 0, 0, 48

    out = bench.adjoint_leg(Args, Lib, _Op(), bench.specs_of(groups), groups, z_all, None)
    for prec in ("fp64", "fp32"):
        assert out[prec]["max_rel_diff_cold"] == 0.0
        assert 0.0 < out[prec]["max_rel_diff_sqrt_checkpoint"] < 1e-13
        assert out[prec]["same_bits_cold_and_sqrt_checkpoint"] is False


def test_a_failing_leg_is_reported():
    def leg():
        raise RuntimeError("no device")
    assert bench.guarded(leg) == {"error": "RuntimeError: no device"}
