"""CPU checks of the drop-in boundary: the C ABI library exports what include/lbm_cuda.h declares,
the extension loads and fails loudly without a GPU, and the host-side helpers behave like the
reference's (python/boltzmann/core.py, python/tests/test_core.py:8-54)."""

import ctypes
import re
import subprocess
from pathlib import Path

import msgpack
import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_symbols() -> set[str]:
    names = set()
    for h in HEADERS:
        text = h.read_text()
        names |= set(re.findall(r"^LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", text, re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for required in ["lbm_create", "lbm_iterate", "lbm_download_fluid", "lbm_upload_f", "lbm_last_error"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    from boltzmann_b200 import LIBRARY

    lib = ctypes.CDLL(str(LIBRARY))
    for name in sorted(declared_symbols()):
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIBRARY)], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (lbm_\w+)", out.stdout))
    assert declared_symbols() <= exported
    # nothing but the declared ABI is exported under the lbm_ prefix
    assert exported == declared_symbols()


def test_abi_version_and_error_without_device():
    from boltzmann_b200 import LIBRARY

    lib = ctypes.CDLL(str(LIBRARY))
    assert lib.lbm_abi_version() == 1
    lib.lbm_last_error.restype = ctypes.c_char_p
    # Argument checks run before any device work.
    counts = (ctypes.c_int64 * 2)(4, 4)
    out = ctypes.c_void_p()
    rc = lib.lbm_create(2, counts, 7, 0, ctypes.c_float(1.0), ctypes.c_float(1.0), 0, ctypes.byref(out))
    assert rc == 1
    assert b"Unknown model: D2Q7" in lib.lbm_last_error()
    rc = lib.lbm_create(4, counts, 9, 0, ctypes.c_float(1.0), ctypes.c_float(1.0), 0, ctypes.byref(out))
    assert rc == 1


def test_extension_classes():
    from boltzmann_b200.core import Omega, PanicException, Simulation, bgk, trt

    assert repr(bgk(0.55)) == "Omega.BGK(1.8181819)"
    o = trt(0.6)
    assert o.kind == "TRT"
    assert np.isclose(o._0, 1 / 0.6) and np.isclose(o._1, 1 / (0.25 / 0.1 + 0.5))
    assert Omega.TRT(1.0, 2.0) == Omega.TRT(1.0, 2.0)
    assert issubclass(PanicException, BaseException) and not issubclass(PanicException, Exception)
    with pytest.raises(PanicException, match="Invalid device type"):
        Simulation("tpu", [4, 4], bgk(0.6))


def test_cell_flags():
    from boltzmann_b200.core import CellFlags

    assert CellFlags.WALL == 1 and CellFlags.FIXED_FLUID == 6 and CellFlags.FIXED_SCALAR_VALUE == 8


def test_check_lbm_params():
    # python/tests/test_core.py:8-18
    from boltzmann_b200.core import check_lbm_params

    with pytest.raises(AssertionError):
        check_lbm_params(1_000_000, 1, tau=0.51)
    with pytest.raises(AssertionError):
        check_lbm_params(1, 1, tau=1.0)
    check_lbm_params(1, 1, tau=0.51)


def test_calc_lbm_params():
    # python/tests/test_core.py:21-54
    from boltzmann_b200.core import calc_lbm_params_lu, calc_lbm_params_si

    tau1, u1 = calc_lbm_params_lu(1, 1)
    tau2, u2 = calc_lbm_params_lu(1, 1, tau=0.51)
    assert tau1 > tau2 and u1 > u2 and abs(tau2 - 0.51) < 1e-8
    assert calc_lbm_params_lu(1, 1, tau=0.51)[1] < calc_lbm_params_lu(10, 1, tau=0.51)[1]
    assert calc_lbm_params_lu(1, 1, tau=0.51)[1] > calc_lbm_params_lu(1, 10, tau=0.51)[1]
    Re, N = 1.0 / 1e-4, 1000
    t1, v1 = calc_lbm_params_lu(Re, N)
    t2, v2 = calc_lbm_params_si(1.0 / N, 1.0, 1.0, 1e-4)
    assert abs(t1 - t2) < 1e-8 and abs(v1 - v2) < 1e-8
    _, v1 = calc_lbm_params_lu(Re, N, tau=0.51)
    _, v2 = calc_lbm_params_si(1.0 / N, 1.0, 1.0, 1e-4, tau=0.51)
    assert abs(v1 - v2) < 1e-8


@pytest.mark.parametrize("dtype", [np.float32, np.int32, np.uint64])
def test_checkpoint_ndarray_encoding_matches_msgpack(dtype):
    """Our vectorised encoder writes what a generic MessagePack library reads back."""
    from boltzmann_b200 import checkpoint as ck

    rng = np.random.default_rng(0)
    if dtype == np.float32:
        a = rng.normal(size=(5, 3, 2)).astype(np.float32)
    elif dtype == np.int32:
        a = rng.integers(-40000, 40000, size=(7, 4)).astype(np.int32)
        a[0, 0] = 3
    else:
        a = np.asarray([4096, 2048, 5], np.uint64)
    w = ck._Writer()
    w.ndarray(a)
    raw = b"".join(w.parts)
    v, dim, data = msgpack.unpackb(raw)
    assert v == 1 and list(dim) == list(a.shape)
    np.testing.assert_array_equal(np.asarray(data, dtype=a.dtype), a.reshape(-1))
    back = ck._Reader(raw).ndarray(dtype)
    np.testing.assert_array_equal(back, a)
    assert back.dtype == dtype


def test_checkpoint_scalars_match_msgpack():
    from boltzmann_b200 import checkpoint as ck

    w = ck._Writer()
    w.array_header(5)
    w.string("tracer")
    w.f32(0.1)
    w.integer(2**40)
    w.integer(-5)
    w.nil()
    out = msgpack.unpackb(b"".join(w.parts))
    assert out[0] == "tracer" and abs(out[1] - 0.1) < 1e-7 and out[2] == 2**40 and out[3] == -5
    assert out[4] is None


def test_checkpoint_velocity_sets_match_oracle():
    from boltzmann_b200 import checkpoint as ck
    from oracle import build as ob
    from oracle.oracle import velocity_set

    ob.build_oracle()
    for d, q in [(1, 3), (2, 9), (2, 5), (3, 7), (3, 27)]:
        ws, qs = ck.velocity_set(d, q)
        c, w, _ = velocity_set(d, q)
        np.testing.assert_array_equal(qs, c)
        np.testing.assert_array_equal(ws, w.astype(np.float32))


def test_lid_driven_cavity_workload():
    from boltzmann_b200 import workloads

    s = workloads.lid_driven_cavities(count=16, lo=20, hi=40, seed=3)
    assert len(s.counts) == 16 and s.cells == sum(a * b for a, b in s.counts)
    for (a, b), sl, tau, re in zip(s.counts, s.domain_slices(), s.tau, s.params["re"]):
        assert 20 <= a <= 40 and a == b
        fl = s.flags[sl].reshape(a, b)
        assert (fl[0] == 1).all() and (fl[-1] == 1).all() and (fl[:, 0] == 1).all()
        assert (fl[1:-1, -1] == 6).all()
        assert (s.vel[sl].reshape(a, b, 2)[1:-1, -1, 0] == np.float32(0.05)).all()
        assert abs(tau - (0.5 + 3 * 0.05 * a / re)) < 1e-12
        assert 100 <= re <= 5000


def test_autotune_cache_key():
    from boltzmann_b200 import autotune

    class Fake:
        counts = [(64, 64), (128, 128), (512, 512)]
        n = 64 * 64 + 128 * 128 + 512 * 512
        collision = 0

    assert autotune.key(Fake(), "f32") == "D2Q9/bgk/f32/cells2^18-width2^7/rows+tiles/rows"
    Fake.counts = [(64, 64), (600, 600)]  # a row over 512 cells: tile kernels only
    Fake.n = 64 * 64 + 600 * 600
    assert autotune.key(Fake(), "f32").endswith("/tiles-only")
