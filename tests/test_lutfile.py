""".radialzlut files: round trip through the C ABI, and ReadLUTFile's per-bead reading
(cputrack/utils.cpp:680-710) of the reference's own fixture files."""
import ctypes as C
import os
from pathlib import Path

import numpy as np
import pytest

from build import SIBLING_REFERENCE  # oracle/build.py: where the reference tree is read from
from qtrk_b200 import lutfile

_REF = Path(os.environ.get("QTRK_REFERENCE") or SIBLING_REFERENCE)
FIXTURES = [_REF / "cputrack-test" / "10x.radialzlut", _REF / "cputrack-test" / "zrange" / "long.radialzlut"]


def test_round_trip(tmp_path, qlib):
    lut = np.random.default_rng(1).normal(size=(3, 20, 16)).astype(np.float32)
    p = tmp_path / "a.radialzlut"
    lutfile.write(p, lut)
    assert p.stat().st_size == 12 + lut.nbytes
    assert np.array_equal(np.frombuffer(p.read_bytes()[:12], np.int32), [3, 20, 16])
    assert np.array_equal(lutfile.read(p), lut)
    b = lutfile.read_bead(f"{p}#2")
    assert b.min() == 0 and abs(b.max() - 1) < 1e-6 and np.allclose(b * (lut[2].max() - lut[2].min()) + lut[2].min(), lut[2], atol=1e-5)
    (tmp_path / "short.radialzlut").write_bytes(p.read_bytes()[:100])
    with pytest.raises(OSError):
        lutfile.read(tmp_path / "short.radialzlut")
    with pytest.raises(OSError):
        lutfile.read(tmp_path / "missing.radialzlut")


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.name)
def test_reference_fixture_files(ref, path):
    if not path.exists():
        pytest.skip("reference fixture file not present")
    lut = lutfile.read(path)
    assert lut.ndim == 3 and lut.shape[0] >= 1
    L = ref.lib
    L.ref_read_lut_file.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.ref_read_lut_file.restype = None
    for k in sorted({0, lut.shape[0] - 1, lut.shape[0] // 2}):
        out = np.zeros(lut.shape[1] * lut.shape[2], np.float32)
        w, h = C.c_int(), C.c_int()
        L.ref_read_lut_file(f"{path}#{k}".encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h))
        assert (h.value, w.value) == lut.shape[1:]
        np.testing.assert_allclose(lutfile.read_bead(f"{path}#{k}"), out.reshape(h.value, w.value), rtol=0, atol=2e-7)
