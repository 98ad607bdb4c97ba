"""The particle-pass autotuner and the histogram layouts it chooses from.

Every configuration must give the reference's result bit for bit (the
layouts only change where the counts are accumulated), and tuning must not
move the beam: tracking after autotune() equals tracking without it.
"""
import numpy as np
import pytest
import torch

from conftest import golden, normwise
from test_gpu_tracking import build, impedance_objects, make_profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import TotalInducedVoltage
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = pytest.mark.gpu


def fused_for(name, **kw):
    g = golden(name)
    ring, rf, beam = build(g)
    prof = make_profile(g, beam)
    ivs = impedance_objects(name, beam, prof, rf)
    tiv = TotalInducedVoltage(beam, prof, ivs) if ivs else None
    return g, beam, FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, **kw)


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
def test_autotune_leaves_the_beam_untouched(cuda, precision):
    g, beam, fx = fused_for("track_full.npz", precision=precision, tune="fixed")
    nt = int(g["n_turns"][0])
    fx.track(nt)
    ref = (fx.dt.cpu().numpy().copy(), fx.dE.cpu().numpy().copy(),
           fx.profile_tensor().cpu().numpy())
    g, beam, fa = fused_for("track_full.npz", precision=precision)
    assert fa.tune_mode == "auto"
    dt0 = fa.dt.cpu().numpy().copy()
    cfg = fa.autotune(reps=2)
    assert cfg["candidates"] > 0 and cfg["particle_pass_ms"] > 0
    # whichever pass wins on this box: every candidate gives the same bits
    assert cfg["kernel"] in ("tma", "plain", "stab", "packed")
    np.testing.assert_array_equal(fa.dt.cpu().numpy(), dt0)
    fa.track(nt)
    np.testing.assert_array_equal(fa.dt.cpu().numpy(), ref[0])
    np.testing.assert_array_equal(fa.dE.cpu().numpy(), ref[1])
    np.testing.assert_array_equal(fa.profile_tensor().cpu().numpy(), ref[2])
    if precision == "f64":
        assert normwise(beam.dt.cpu().numpy(), g["dt"]) < 1e-11


@pytest.mark.parametrize("kernel", ["tma", "plain"])
@pytest.mark.parametrize("hist", [-1, 0, 1, 2, 3])
def test_every_histogram_layout_matches_reference(cuda, kernel, hist):
    g, beam, f = fused_for("track_full.npz", precision="f64", kernel=kernel)
    f.eng.call("set_histogram", hist)
    nt = int(g["n_turns"][0])
    f.track(nt)
    assert normwise(beam.dt.cpu().numpy(), g["dt"]) < 1e-11
    assert normwise(beam.dE.cpu().numpy(), g["dE"]) < 1e-11
    np.testing.assert_array_equal(f.profile_tensor().cpu().numpy(), g["profiles"][-1])


def test_autotuned_tracker_is_the_default(cuda):
    g, beam, f = fused_for("track_rf.npz")
    assert f.tuned is None
    f.track(int(g["n_turns"][0]))
    assert f.tuned is not None
    assert normwise(beam.dt.cpu().numpy(), g["dt"]) < 1e-11
    np.testing.assert_array_equal(f.profile_tensor().cpu().numpy(), g["profiles"][-1])


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
@pytest.mark.parametrize("stages", [2, 4])
@pytest.mark.parametrize("hist", [0, 1, 3])
def test_prefetch_ring_matches_direct_loads(cuda, precision, stages, hist):
    g, beam, fx = fused_for("track_full.npz", precision=precision, kernel="plain")
    nt = int(g["n_turns"][0])
    fx.track(nt)
    ref = (fx.dt.cpu().numpy().copy(), fx.dE.cpu().numpy().copy(),
           fx.profile_tensor().cpu().numpy())
    g, beam, f = fused_for("track_full.npz", precision=precision, kernel="plain")
    f.eng.call("set_prefetch", stages)
    f.eng.call("set_histogram", hist)
    f.track(nt)
    np.testing.assert_array_equal(f.dt.cpu().numpy(), ref[0])
    np.testing.assert_array_equal(f.dE.cpu().numpy(), ref[1])
    np.testing.assert_array_equal(f.profile_tensor().cpu().numpy(), ref[2])


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
@pytest.mark.parametrize("cluster", [2, 4])
@pytest.mark.parametrize("hist", [0, 1])
def test_cluster_merged_histograms_match(cuda, precision, cluster, hist):
    g, beam, fx = fused_for("track_full.npz", precision=precision, kernel="plain")
    nt = int(g["n_turns"][0])
    fx.track(nt)
    ref = (fx.dt.cpu().numpy().copy(), fx.profile_tensor().cpu().numpy())
    g, beam, f = fused_for("track_full.npz", precision=precision, kernel="plain")
    f.eng.call("set_cluster", cluster)
    f.eng.call("set_histogram", hist)
    f.eng.call("set_prefetch", 2)
    f.track(nt)
    np.testing.assert_array_equal(f.dt.cpu().numpy(), ref[0])
    np.testing.assert_array_equal(f.profile_tensor().cpu().numpy(), ref[1])


@pytest.mark.parametrize("precision", ["f64", "f32p64", "q32p64"])
@pytest.mark.parametrize("ring,l2", [(0, 0), (2, 0), (2, 1)])
def test_shared_table_pass_gives_the_global_table_bits(cuda, precision, ring, l2):
    """The plain pass with the table in shared memory (the induced voltage
    only for F64 / Q32P64, entries formed per particle; the float2 table
    for F32P64) and a packed histogram, at C2's 2^14 slices on 2e6
    particles: the same bits as the plain pass over the global table."""
    import bench
    out = []
    for kernel in ("plain", "stab"):
        fused, beam, _ = bench.build_fused(2_000_000, 16384, 4, precision, kernel=kernel)
        fused.eng.call("set_prefetch", ring if kernel == "stab" else 2)
        fused.eng.call("set_l2_prefetch", l2 if kernel == "stab" else 0)
        fused.eng.call("tune", 1024, 1, 2)
        fused.track(4)
        fused.check()
        out.append((fused.dt.cpu().numpy(), fused.dE.cpu().numpy(),
                    fused.profile_tensor().cpu().numpy(),
                    fused.induced_voltage_tensor().cpu().numpy()))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("precision", ["f64", "f32p64", "q32p64"])
@pytest.mark.parametrize("slices,ring", [(16384, 0), (16384, 4), (65536, 0), (65536, 2)])
def test_packed_histogram_pass_gives_the_plain_pass_bits(cuda, precision, slices, ring):
    """The plain pass with a packed 16-bit block histogram over the global
    table (the form that fits 2^16-slice profiles beside its ring), on 2e6
    particles: the same bits as the plain pass with its int32 histogram."""
    import bench
    out = []
    for kernel in ("plain", "packed"):
        fused, beam, _ = bench.build_fused(2_000_000, slices, 4, precision, kernel=kernel)
        fused.eng.call("set_prefetch", ring if kernel == "packed" else 0)
        fused.eng.call("tune", 1024, 1, 2)
        fused.track(4)
        fused.check()
        out.append((fused.dt.cpu().numpy(), fused.dE.cpu().numpy(),
                    fused.profile_tensor().cpu().numpy(),
                    fused.induced_voltage_tensor().cpu().numpy()))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("slices", [16384, 65536])
def test_overlap_tuning_restores_the_turn_state(cuda, slices):
    """The autotuner's whole-turn replays (overlap on and off) start from
    and return to the run's state: coordinates, profile, induced voltage
    and turn counter; tracking afterwards gives the untuned run's bits."""
    import bench
    runs = []
    for tune in ("auto", "fixed"):
        fused, beam, _ = bench.build_fused(1_000_000, slices, 40, "f64")
        if tune == "fixed":
            fused.eng.call("tune", 1024, 1, 5)
            fused.tune_mode = "fixed"
        fused.track(2)
        fused.sync()
        before = (fused.dt.cpu().numpy().copy(), fused.profile_tensor().cpu().numpy(),
                  fused.induced_voltage_tensor().cpu().numpy())
        if tune == "auto":
            cfg = fused.autotune(reps=1)
            assert "overlap" in cfg
            fused.sync()
            after = (fused.dt.cpu().numpy(), fused.profile_tensor().cpu().numpy(),
                     fused.induced_voltage_tensor().cpu().numpy())
            for x, y in zip(before, after):
                np.testing.assert_array_equal(x, y)
        fused.track(10)
        fused.check()
        runs.append((fused.dt.cpu().numpy(), fused.dE.cpu().numpy(),
                     fused.profile_tensor().cpu().numpy(),
                     fused.induced_voltage_tensor().cpu().numpy()))
    for x, y in zip(*runs):
        np.testing.assert_array_equal(x, y)


def test_overlap_off_gives_the_same_bits(cuda):
    import bench
    out = []
    for on in (1, 0):
        fused, beam, _ = bench.build_fused(1_000_000, 16384, 8, "f64", kernel="stab")
        fused.eng.call("set_overlap", on)
        fused.eng.call("tune", 1024, 1, 3)
        fused.track(8)
        fused.check()
        out.append((fused.dt.cpu().numpy(), fused.dE.cpu().numpy(),
                    fused.profile_tensor().cpu().numpy(),
                    fused.induced_voltage_tensor().cpu().numpy()))
    for x, y in zip(*out):
        np.testing.assert_array_equal(x, y)


def test_shared_table_pass_is_refused_where_it_does_not_apply(cuda):
    from blond_b200 import BlondB200Error
    g, beam, f = fused_for("track_rf.npz", precision="f64", kernel="stab")
    with pytest.raises(BlondB200Error, match="shared-table"):
        f.track(1)
    g, beam, f = fused_for("track_rf.npz", precision="f64", kernel="packed")
    with pytest.raises(BlondB200Error, match="packed-histogram"):
        f.track(1)
