"""The bench line's bookkeeping, checked on the CPU: the byte model of the
roofline (the survey's compulsory bytes at the 3.6 M-tet configuration),
the DRAM traffic read from the committed ncu summary, the peak fallback,
the workload description shared by both arms, and the defaults of a plain
`python bench.py` run (timing rules: at least 3 warm-up steps, at least 200
timed steps)."""

import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO))

import bench  # noqa: E402

# 200 x 60 x 50 Kuhn channel
C2 = {"n_tets": 3_600_000, "n_nodes": 625_311, "nnz": 9_175_931}


def test_byte_model_at_the_bench_configuration():
    bm = bench.bytes_model(C2)
    E, N, Z = C2["n_tets"], C2["n_nodes"], C2["nnz"]
    # element sweep 164 E + 32 N, row gather 64 E + 8 N + 8 Z
    assert bm["elem_sweep"] == 164 * E + 32 * N == 610_409_952
    assert bm["row_gather"] == 64 * E + 8 * N + 8 * Z
    assert bm["fused"] == bm["elem_sweep"] + bm["row_gather"] == 919_219_888
    assert bm["term3"] == 0
    assert bench.bytes_model(C2, n_active=10)["term3"] == 10 * 16 * 16
    # this layout's own bytes: B and V recomputed, displacements and the
    # local-matrix round trip added
    assert bm["design"]["elem_sweep"] == E * 245 + N * 32


def test_traffic_from_the_committed_profile():
    # 229.3 B per element measured on the 1.62 M-tet capture, scaled
    assert bench.read_traffic("elem_sweep", C2["n_tets"]) == pytest.approx(825_480_000, rel=1e-9)
    assert bench.read_traffic("no_such_kernel", C2["n_tets"]) is None


def test_peak_source_is_named():
    peak, kind = bench.read_peaks()
    assert kind in ("measured", "fallback") and peak > 1000.0
    if kind == "fallback":
        assert peak == 6650.0


def test_workload_description_has_no_model_keys():
    class M:
        n_tets, n_nodes = C2["n_tets"], C2["n_nodes"]
    d = bench.config_dict((200, 60, 50), M)
    assert d["workload"].startswith("transonic bump channel 200x60x50")
    assert "model" not in d and "global_batch" not in d and "seq_len" not in d
    assert d["mesh"] == "200x60x50" and d["states"] == bench.N_STATES


def test_plain_run_defaults(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.impl != "reference"
    assert a.warmup >= 3 and a.steps >= 200
    assert a.cpu_states >= 1
