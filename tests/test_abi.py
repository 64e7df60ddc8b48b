"""The C-ABI library loads, exports every entry point include/cfs.h declares,
validates configurations on the host, and has no CPU path (no GPU compute here)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "cfs.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfs_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_entry_point_is_exported_and_bound(cfsb):
    lib = cfsb.load_library()
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(cfsb.exported_symbols()) == declared


def test_abi_version_and_defaults(cfsb):
    lib = cfsb.load_library()
    assert lib.cfs_abi_version() == 3
    import ctypes
    cfg = cfsb.CfsConfig()
    lib.cfs_config_default(ctypes.byref(cfg))
    assert cfg.gamma == 1.4 and cfg.weno_eps == 1e-2
    assert cfg.rk == cfsb.RK_TVD3_REFERENCE and cfg.hll == cfsb.HLL_REFERENCE
    assert list(cfg.bc) == [cfsb.BC_NEUMANN] * 4
    assert cfg.rounding == cfsb.ROUND_STOCHASTIC_ALL and cfg.march_rows == 0


@pytest.mark.parametrize("kw,msg", [
    (dict(nx=2), "at least 3"),
    (dict(lx=-1.0), "positive"),
    (dict(bc=(2, 0, 0, 0)), "pairs"),
    (dict(precision=7), "precision"),
    (dict(weno_eps=0.0), "weno_eps"),
    (dict(bc=(1, 0, 0, 0), bc_prim=[[0.0, 0, 0, 1]] * 4), "density"),
])
def test_invalid_configs_are_rejected_on_the_host(cfsb, kw, msg):
    args = dict(nx=16, ny=16)
    args.update(kw)
    nx, ny = args.pop("nx"), args.pop("ny")
    with pytest.raises(cfsb.CfsError) as e:
        cfsb.Solver(nx, ny, **args)
    assert e.value.code == 1 and msg in str(e.value)


def test_no_cpu_fallback_without_a_device(cfsb):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(cfsb.CfsError) as e:
        cfsb.Solver(16, 16)
    assert e.value.code == 2


def test_gpu_plugin_harness_links_the_product_library():
    """oracle/_ref/libref_gpu.so (reference classes + GPU plugins) loads on a
    host without a GPU and exports its entry point; it resolves libcfs.so
    from the package directory."""
    import oracle_bind as ob
    if not ob.REF_GPU.exists():
        pytest.skip("built only where the reference tree is")
    lib = ob.ref_gpu_lib()
    assert hasattr(lib, "ref_gpu_run")
