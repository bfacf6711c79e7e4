"""Builder parity at the benchmarked sizes: the product's CB structure of the
full power-law (n = 2^20, 16.8M stored values) and stencil (64^3 x 3 dof,
61.7M) workloads equals, array by array and bit for bit, the structure the
reference's own host code builds from the same COO (oracle/_ref, compiled from
the reference's headers).  Also pins the headline workload's algorithmic byte
count, which the bench's reference arm uses without loading the library."""
import gc
import importlib.util
import pathlib

import pytest

import cbdump as cd

pytestmark = pytest.mark.skipif(not cd.have_ref(), reason="oracle/_ref not built")


def _bench_constant():
    spec = importlib.util.spec_from_file_location(
        "bench_consts", pathlib.Path(__file__).resolve().parent.parent / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.PL_FP64_ALG_BYTES


@pytest.mark.parametrize("name", ["pl", "st"])
def test_fullsize_builder_matches_reference(name):
    import cbspmv
    from cbspmv import gen
    coo = gen.power_law() if name == "pl" else gen.stencil_27pt()
    ref = cd.ref_build(coo, 16, 1)
    plan = cbspmv.Plan(coo)
    cd.compare_dumps(ref, plan.export(), f"{name} full size")
    if name == "pl":
        assert plan.info()["algorithmic_bytes"] == _bench_constant()
    del ref, plan
    gc.collect()
