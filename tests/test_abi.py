"""C ABI: the library loads and exports every symbol include/rabung_census.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import re

from conftest import ROOT


def declared():
    h = (ROOT / "include" / "rabung_census.h").read_text()
    body = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    return sorted(set(re.findall(r"\b(cz_[a-z0-9_]+|baseline_[a-z]+)\s*\(", body)))


def test_header_symbols_exported():
    from rabung_atlas32_b200 import build, _lib
    build.build()
    lib = ctypes.CDLL(str(build.LIB))
    names = declared()
    assert "cz_census" in names and "baseline_profile" in names
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.EXPORTS)


def test_struct_layouts():
    from rabung_atlas32_b200 import _lib
    assert ctypes.sizeof(_lib.cz_profile) == 32
    assert ctypes.sizeof(_lib.cz_config) == 4 * (1 + 1 + 1 + 10 + 1 + 1 + 1 + 1 + 1 + 1 + 1 + 10 + 1 + 1 + 10 + 1)


def test_count_profiles_host_only():
    from rabung_atlas32_b200 import _lib, codec
    lib = _lib.load()
    ps = [2, 3, 5, 7, 4294967291]
    arr = (ctypes.c_uint32 * len(ps))(*ps)
    assert lib.cz_count_profiles(arr, len(ps)) == sum(bin(codec.expected_mask(p)).count("1") for p in ps[1:])


def test_default_config_and_bad_tuning_refused_before_device():
    """cz_default_config fills the measured per-order anchor stages; cz_open
    validates a tuning before it looks for a device, so a bad one is refused
    with CZ_EINVAL on any host."""
    from rabung_atlas32_b200 import _lib
    from rabung_atlas32_b200.census import Tuning
    lib = _lib.load()
    cfg = _lib.cz_config()
    assert lib.cz_default_config(ctypes.byref(cfg)) == _lib.CZ_OK
    assert tuple(cfg.anchor_t) == Tuning().anchor_t
    assert tuple(cfg.q_cap) == Tuning().q_cap and tuple(cfg.spec_margin10) == Tuning().spec_margin10
    h = ctypes.c_void_p()
    for field, r, bad in [("anchor_t", 5, 1), ("anchor_t", 2, 33), ("q_cap", 3, 2), ("q_cap", 9, 256)]:
        lib.cz_default_config(ctypes.byref(cfg))
        getattr(cfg, field)[r] = bad
        assert lib.cz_open(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CZ_EINVAL, (field, r, bad)
    lib.cz_default_config(ctypes.byref(cfg))
    cfg.cover_n = 1
    assert lib.cz_open(ctypes.byref(cfg), ctypes.byref(h)) == _lib.CZ_EINVAL


def test_count_profiles64_host_only():
    """The wide count needs no GPU; primes at or above 2^33 give 0."""
    from rabung_atlas32_b200 import _lib, codec
    lib = _lib.load()
    ps = [3, 4294967311, 5389000007, 8589934583]
    arr = (ctypes.c_uint64 * len(ps))(*ps)
    assert lib.cz_count_profiles64(arr, len(ps)) == sum(bin(codec.expected_mask(p)).count("1") for p in ps)
    big = (ctypes.c_uint64 * 1)(2 ** 33 + 17)
    assert lib.cz_count_profiles64(big, 1) == 0
    assert ctypes.sizeof(_lib.cz_profile64) == 40
