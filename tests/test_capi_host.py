"""CPU-only checks: the C-ABI library loads and exports every declared symbol,
status codes map to the reference's exceptions, the C oracle agrees with
the numpy oracle, and the workload generators follow the unit mapping."""
import ctypes
import os

import numpy as np
import pytest

from energy_level_b200 import _lib, configs
from energy_level_b200.build import build
from oracle import ref


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.load()


def test_library_exports_every_header_function(lib):
    names = _lib.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the binding table covers the header exactly
    assert sorted(_lib.PROTOTYPES) == names


def test_library_is_sm100a_only():
    # every CUDA source is built for sm_100a and nothing else
    from energy_level_b200 import build as b
    assert b.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_version_and_null_context(lib):
    assert lib.el_version() >= 100
    assert lib.el_last_error(None) == b"null context"
    assert lib.el_ctx_launches(None) == -1
    # no device in this container: context creation reports a CUDA error, never crashes
    h = ctypes.c_void_p()
    rc = lib.el_ctx_create(0, None, ctypes.byref(h))
    assert rc in (_lib.EL_OK, _lib.EL_ECUDA)
    if rc == _lib.EL_OK:
        lib.el_ctx_destroy(h)


def test_status_mapping():
    with pytest.raises(ValueError):
        _lib.check(_lib.EL_EINVAL)
    with pytest.raises(MemoryError):
        _lib.check(_lib.EL_ENOMEM)
    with pytest.raises(RuntimeError, match="用户取消"):
        _lib.check(_lib.EL_ECANCEL)
    with pytest.raises(RuntimeError):
        _lib.check(_lib.EL_ECUDA)
    _lib.check(_lib.EL_OK)


def test_c_oracle_matches_numpy_oracle():
    from oracle import build as ob
    n = 9
    rng = np.random.default_rng(11)
    om = rng.uniform(0.5, 2.0, n)
    de = rng.uniform(-3, 3, n)
    pairs = configs.pairs_from_positions(configs.chain_positions(n))
    d = ob.diag_full(n, de, pairs)
    assert np.allclose(d, ref.diagonal(n, np.arange(1 << n), de, pairs), atol=1e-12, rtol=0)
    H = ref.dense_h(n, None, om, de, pairs)
    _, _, c, r = ref.kpm_bounds(H)
    z = rng.choice(np.array([-1, 1], dtype=np.int8), size=(3, 1 << n))
    m1 = ob.kpm_full(n, om, d, c, r, 30, z)
    m2 = ref.kpm_moments(lambda v: H @ v, 1 << n, 30, z, c, r)
    assert np.max(np.abs(m1 - m2)) < 1e-12


def test_workload_unit_mapping():
    c1 = configs.chain12()
    assert c1["n"] == 12 and np.all(c1["delta"] == -1.0) and np.all(c1["Om"] == 2.0)
    V01 = c1["calib"]["pairs"][0]["V"]
    assert abs(V01 - 862690.0 / 5.5 ** 6) < 1e-9
    c2 = configs.square25()
    assert len(c2["calib"]["pairs"]) == 300 and c2["num"] == 1024 and c2["nvec"] == 32
    assert np.all(np.abs(c2["delta"]) <= 3.0)
    c3 = configs.chain31()
    assert len(c3["segments"]) == 300 and len(c3["calib"]["pairs"]) == 465
    assert c3["segments"][0]["delta"][0] == 6.0     # delta = -Delta, Delta starts at -6
    c4 = configs.batch512(count=16)
    assert all(16 <= c["n"] <= 22 for c in c4)
    c5 = configs.ring20()
    assert len(c5["omega_k"]) == 200 and c5["target"].startswith("rgrg")


def test_counter_probes_are_rademacher_and_stable():
    from energy_level_b200.probes import rademacher_host
    z = rademacher_host(seed=2, probe0=0, nvec=4, dim=1000)
    assert set(np.unique(z)) == {-1, 1}
    assert abs(z.mean()) < 0.1
    assert np.array_equal(z, rademacher_host(seed=2, probe0=0, nvec=4, dim=1000))
    assert np.array_equal(z[2:], rademacher_host(seed=2, probe0=2, nvec=2, dim=1000))
