"""The bounds-checked build: every kernel family, run through libqcb_checked.so on small and
ragged lattices, forms no field index outside its field; and the check itself works.

compute-sanitizer is not available for this purpose, so the library carries its own check
(QCB_CHECKED): each (mu, parity, h) a link or algebra access is formed from is validated on the
device, counted and recorded when bad, and the access redirected inside the field.  The workload
runs in a subprocess (tests/checked_workload.py) because the binding binds one library per
process.  The positive control sends two links outside a 4^4 field (h = V/2 + 3, and mu = 5)
through qcb_debug_probe_link; the normal build refuses those on the host, the checked build must
count each once and record its (kind, mu, parity, h).
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def report():
    r = subprocess.run([sys.executable, os.path.join(HERE, "checked_workload.py")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-4000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_no_out_of_bounds_access(report):
    assert report["checked"] is True
    assert report["count"] == 0, hex(report["first"])


def test_checked_build_catches_probes(report):
    a, b = report["probes"]
    assert a["count"] == 1 and (a["kind"], a["mu_rec"], a["par_rec"], a["h_rec"]) == (0, 0, 1, 128 + 3)
    assert b["count"] == 1 and (b["kind"], b["mu_rec"], b["par_rec"], b["h_rec"]) == (0, 5, 0, 7)
    # a redirected load reads a valid link and writes nothing into the field
    assert report["plaquette_after_probes"] == report["plaquette_before_probes"]


def test_normal_build_refuses_probe_outside_field(gpu):
    f = gpu.GaugeField((4, 4, 4, 4), 64, 0)
    f.hot_start(1)
    f.debug_probe_link(3, 1, 127)  # the last link of the field: accepted
    for mu, par, h in [(0, 1, 128 + 3), (5, 0, 7), (0, 2, 0), (0, 0, -1)]:
        with pytest.raises(gpu.QcbError) as e:
            f.debug_probe_link(mu, par, h)
        assert e.value.code == -1
    assert gpu.debug_oob() == (False, 0, 0)
