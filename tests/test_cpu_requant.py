"""The re-encoders' shift form of requantization (lossy stored bins moved to
the request or residual bounds with an integer shift) equals the composition
of the reference's quantizers (d_iSQ_IABS_4 -> d_CQ_IABS_4 for init_send,
d_RESI_4.h:57-76 for resi_send), checked over every lossy bin for a few
exponent sets and over a dense sample for the rest."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "requant_check.c")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    from oracle import oracle as O
    lib = O.build()
    exe = str(tmp_path_factory.mktemp("rq") / "requant_check")
    subprocess.check_call(["gcc", "-O2", "-fopenmp", "-o", exe, SRC, "-L", os.path.dirname(lib),
                           "-lcortado_oracle", "-Wl,-rpath," + os.path.dirname(lib)])
    return exe


def _run(exe, mode, es, e1, e2, full):
    r = subprocess.run([exe, str(mode), str(es), str(e1), str(e2), str(int(full))], capture_output=True, text=True,
                       timeout=600)
    checked, fastn, bad = (int(v) for v in r.stdout.split())
    return r.returncode, checked, fastn, bad


KS = (0, 1, 2, 3, 7, 12, 22, 23, 24, 25, 31, 33)


@pytest.mark.parametrize("es", (1, 100, 190))
def test_init_send_shift_form(checker, es):
    for k1 in KS:
        rc, checked, fastn, bad = _run(checker, 0, es, es + k1, 1, full=(k1 in (0, 1, 7) and es == 100))
        assert bad == 0 and rc == 0, (es, k1)
        assert fastn > 0


@pytest.mark.parametrize("es", (1, 100, 190))
def test_resi_send_shift_form(checker, es):
    for k1 in KS:
        for k2 in KS:
            if k2 > k1:
                continue
            rc, checked, fastn, bad = _run(checker, 1, es, es + k1, es + k2, full=((k1, k2) in ((2, 1), (7, 0), (12, 3)) and es == 100))
            assert bad == 0 and rc == 0, (es, k1, k2)
            assert fastn > 0
