"""The host-native build of the FP32 oracle (test infrastructure, CPU only).

The CPU baseline of bench.py times the oracle compiled with -march=native on
the host that runs it.  It keeps the portable build's rounding flags
(-ffp-contract=off, no fast math), so its steps must give bit-identical
particles; checked here on two scenes after a few steps."""
import numpy as np
import pytest

from nexus_b200 import scenes


@pytest.mark.parametrize("name", ["cube", "sandwater"])
def test_native_oracle_matches_portable_bit_for_bit(oracle_built, name):
    from oracle.oracle import OracleScene, native_path
    if native_path() is None:
        pytest.skip("no compiler for a host-native build here")
    sc = scenes.elastic_cube(n_side=10, steps=5) if name == "cube" else scenes.sand_water(scale=0.05, steps=5)
    a, b = OracleScene(sc, "f32"), OracleScene(sc, "f32", native=True)
    assert a.L is not b.L and b.L.oracle_path != a.L.oracle_path
    a.step(5)
    b.step(5)
    pa, pb = a.particles(), b.particles()
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), k
