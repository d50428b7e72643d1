"""bench.py's workload generators still produce the simulations the oracle fixtures were made from
(CPU only; the GPU lines compare their results with those fixtures and would otherwise report
parity as not checked or fail): the uneven batch's draw has the fixture's spec digest, and the
49^3 sweep has 3,742,848 simulations whose every-64th sample is the one the fixture holds."""
import hashlib
import json
import os

import numpy as np

import bench

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# SHA-256 of bench.sweep_descs(49, 32, (2, 3, 4, 5))[::64] (SIM_DESC_DTYPE records) when
# tests/golden/sweep49_fixture.json was made
SWEEP49_SAMPLE_SHA256 = "ec71f3f1318d7f661cd381b5bfa3c8817597d44a61077df321887ef83f9f9169"


def test_uneven_batch_draw_matches_its_fixture():
    fx = json.load(open(os.path.join(GOLDEN, "engine_fixture.json")))["uneven"]
    sims = bench.uneven_sims(fx["sims"])
    assert len(sims) == fx["sims"] == 2048
    assert bench.uneven_spec_digest(sims) == fx["spec_sha256"]
    assert {s["edge"] for s in sims} <= {33, 49, 65, 97, 129, 193}


def test_sweep49_sample_matches_its_fixture():
    fx = json.load(open(os.path.join(GOLDEN, "sweep49_fixture.json")))
    full = bench.sweep_descs(49, 32, (2, 3, 4, 5))
    assert len(full) == fx["sims_total"] == 3742848
    sample = np.ascontiguousarray(full[::fx["stride"]])
    assert len(sample) == fx["sims"]
    assert hashlib.sha256(sample.tobytes()).hexdigest() == SWEEP49_SAMPLE_SHA256
    assert fx["viable"] + fx["possible"] + fx["unviable"] == fx["sims"]
