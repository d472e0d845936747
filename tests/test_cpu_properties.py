"""Property tests (hypothesis) of host logic that hand-picked cases cover thinly.

* ``rust_exp`` reproduces Rust's ``{:20.12e}`` layout of an f64 (the ENERTRJ
  writer, crates/gromos-io/src/energy.rs:181-460): a 13-digit mantissa, an
  exponent without sign padding or leading zeros, right-aligned in 20
  columns, and the value survives the round trip to 12 significant digits;
* energy frames written by ``EnergyWriter`` read back to the same values;
* ``shard_by_work`` partitions the systems completely, deterministically and
  within the greedy longest-first bound.
"""
import re

import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

from gromos_nb import gromos_io as io
from gromos_nb.replicas import shard_by_work

FINITE = st.floats(allow_nan=False, allow_infinity=False, width=64)
RUST_E = re.compile(r"^-?\d\.\d{12}e-?(0|[1-9]\d*)$")


@settings(max_examples=400, deadline=None)
@given(FINITE)
def test_rust_exp_layout_and_round_trip(x):
    s = io.rust_exp(x)
    t = s.lstrip(" ")
    assert len(s) == max(20, len(t))
    assert RUST_E.match(t), s
    mant, exp = t.split("e")
    assert float(t) == float(f"{x:.12e}")            # the same correctly rounded 13 digits
    assert abs(float(mant)) < 10.0 and (float(mant) == 0.0 or abs(float(mant)) >= 1.0)
    assert int(exp) == int(f"{x:.12e}".split("e")[1])  # same exponent, printed without sign padding


@settings(max_examples=40, deadline=None)
@given(st.lists(st.tuples(st.floats(0.0, 1e6), st.floats(-1e6, 1e6), st.integers(0, 10**6)),
                min_size=1, max_size=5))
def test_energy_frames_round_trip(tmp_path_factory, rows):
    path = str(tmp_path_factory.mktemp("tre") / "e.tre")
    frames = [io.md_energy_frame(0.002 * k, kin, pot, pot * 0.25, n_dof, volume=27.0)
              for k, (kin, pot, n_dof) in enumerate(rows)]
    with io.EnergyWriter(path, "property") as w:
        for f in frames:
            w.write_frame(f)
    back = io.read_energy_trajectory(path)
    assert len(back) == len(frames)
    for a, b in zip(frames, back):
        np.testing.assert_allclose(b.values(), a.values(), rtol=1e-12, atol=1e-300)


@settings(max_examples=200, deadline=None)
@given(st.lists(st.floats(0.0, 1e6), min_size=0, max_size=60), st.integers(1, 9))
def test_shard_by_work_partition_and_bound(work, world):
    shards = shard_by_work(work, world)
    assert len(shards) == world
    assert sorted(i for s in shards for i in s) == list(range(len(work)))
    assert all(s == sorted(s) for s in shards)
    assert shard_by_work(work, world) == shards
    loads = [sum(work[i] for i in s) for s in shards]
    if work:
        assert max(loads) - min(loads) <= max(work) * (1 + 1e-12) + 1e-9
