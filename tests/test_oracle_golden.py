"""Pins the CPU oracle to the reference: replays every golden case through the
oracle and compares stream and decoded-file hashes with those the reference's
own binaries produced on a B200 (tests/golden/reference_outputs.json)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G


class OracleImpl:
    def noa_range(self, x):
        return np.nanmin(x), np.nanmax(x)

    def store(self, x, eb):
        return O.store_encode(x, eb)

    def init_send(self, stored, n, eb):
        return O.init_send(stored, eb)

    def init_recv(self, s):
        return O.init_recv(s)

    def resi_send(self, stored, n, src, dst):
        return O.resi_send(stored, src, dst)

    def resi_recv(self, src, s):
        return O.resi_recv(src, s)


REF = G.reference_outputs()
CASES = [(n, s) for n, s in G.cases()] + [("c1_sin128", G.c1_setting())]


@pytest.mark.parametrize("name,setting", CASES, ids=[f"{n}-{s['tag']}" for n, s in CASES])
def test_oracle_matches_reference(name, setting):
    key = f"{name}/{setting['tag']}"
    ref = REF[key]
    x = G.load_input(name)
    if x is None:
        pytest.skip("synthetic input not bit-reproducible on this machine")
    rec = G.run_flow(OracleImpl(), x, setting)
    diffs = G.compare(rec, ref)
    assert not diffs, diffs
