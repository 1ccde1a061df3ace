"""Body commands on the CPU: the oracle's restatement of body_edits.wgsl, and the boundary.

crates/dynamis-rigid/shaders/body_edits.wgsl:35-103 runs each body's queued commands in order
after clear_inputs.wgsl and before activity.wgsl (crates/dynamis-rigid/src/apply_commands.rs:
273-293). The oracle's restatement is pinned on behaviours: an impulse changes the velocity by
impulse / mass, a force acts for one step only, a patch teleports, sleep freezes and counts,
wake counts, and commands on one body compose in the order given.
"""
import numpy as np
import pytest

from dynamis_b200 import DynamisError, World, scenes
from dynamis_b200 import records as R
from oracle.oracle import oracle_from_world

DT = 1.0 / 60.0


def random_edits(rng, ids, count, extent=4.0):
    """`count` commands of every kind on bodies drawn from `ids` (repeats allowed)."""
    recs = np.zeros(count, R.BODY_EDIT)
    who = rng.choice(np.asarray(ids), size=count)
    kinds = rng.integers(0, 9, size=count)
    for i, kind in enumerate(kinds):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        recs[i] = R.body_edit(int(kind), mask=int(rng.integers(1, 16)),
                              position=rng.uniform(-extent / 2, extent / 2, 3) + (0.0, extent / 2 + 0.6, 0.0),
                              orientation=q, velocity=rng.normal(0.0, 2.0, 3), angular_velocity=rng.normal(0.0, 1.0, 3),
                              force=rng.normal(0.0, 60.0, 3), torque=rng.normal(0.0, 10.0, 3))[0]
    return who.astype(np.uint32), recs


def floating_sphere():
    w = World()
    ids = scenes.sphere_row(1).build(w)
    o = oracle_from_world(w, DT)
    inverse_mass = float(w.export_scene()["descs"]["inverse_mass"][0])
    return w, o, int(ids[0]), inverse_mass


def test_an_impulse_changes_the_velocity_by_impulse_over_mass():
    w, o, body, im = floating_sphere()
    o.edit_bodies([body], R.body_edit(R.EDIT_IMPULSE, velocity=(3.0, 0.0, -1.0)))
    o.step(DT)
    v = o.states()["velocity"][0]
    assert np.allclose(v, np.array([3.0, 0.0, -1.0]) * im, rtol=1e-3)
    o.close()
    w.close()


def test_a_force_acts_for_one_step():
    w, o, body, im = floating_sphere()
    o.edit_bodies([body], R.body_edit(R.EDIT_FORCE, force=(0.0, 0.0, 120.0)))
    o.step(DT)
    v1 = o.states()["velocity"][0].copy()
    assert np.isclose(v1[2], 120.0 * im * DT, rtol=1e-3)
    o.step(DT)
    assert np.allclose(o.states()["velocity"][0], v1, rtol=1e-3)  # cleared at the next step
    o.close()
    w.close()


def test_a_force_off_the_centre_spins_the_body():
    w, o, body, _ = floating_sphere()
    centre = o.states()["position"][0]
    o.edit_bodies([body], R.body_edit(R.EDIT_FORCE_AT_POINT, force=(0.0, 50.0, 0.0), position=centre + (0.5, 0.0, 0.0)))
    o.step(DT)
    spin = o.states()["angular_velocity"][0]
    assert spin[2] > 0.0 and abs(spin[0]) < 1e-6 and abs(spin[1]) < 1e-6
    o.close()
    w.close()


def test_a_patch_teleports_the_body():
    w, o, body, _ = floating_sphere()
    o.edit_bodies([body], R.body_edit(R.EDIT_PATCH, mask=R.PATCH_POSITION, position=(10.0, 2.0, -3.0)))
    o.step(DT)
    assert np.array_equal(o.states()["position"][0], np.float32([10.0, 2.0, -3.0]))
    o.close()
    w.close()


def test_sleep_freezes_and_wake_releases_with_counts():
    w, o, body, im = floating_sphere()
    o.edit_bodies([body], R.body_edit(R.EDIT_IMPULSE, velocity=(1.0, 0.0, 0.0)))
    o.step(DT)
    o.edit_bodies([body], R.body_edit(R.EDIT_SLEEP))
    o.step(DT)
    s = o.states()[0]
    assert s["sleeping"] == 1 and not s["velocity"].any()
    assert o.counters()[R.COUNTER["SLEPT"]] == 1
    at_rest = s["position"].copy()
    o.step(DT)
    assert np.array_equal(o.states()["position"][0], at_rest)
    o.edit_bodies([body], R.body_edit(R.EDIT_WAKE))
    o.step(DT)
    assert o.states()["sleeping"][0] == 0
    assert o.counters()[R.COUNTER["WOKE"]] == 1
    o.close()
    w.close()


def test_commands_on_one_body_run_in_order():
    w, o, body, im = floating_sphere()
    patch = R.body_edit(R.EDIT_PATCH, mask=R.PATCH_VELOCITY, velocity=(1.0, 0.0, 0.0))
    push = R.body_edit(R.EDIT_IMPULSE, velocity=(0.0, 0.0, 2.0))
    o.edit_bodies([body, body], np.concatenate([patch, push]))
    o.step(DT)
    assert np.allclose(o.states()["velocity"][0], [1.0, 0.0, 2.0 * im], rtol=1e-3)
    o.edit_bodies([body, body], np.concatenate([push, patch]))
    o.step(DT)
    assert np.allclose(o.states()["velocity"][0], [1.0, 0.0, 0.0], rtol=1e-3)  # the patch overwrote the push
    o.close()
    w.close()


def test_random_commands_keep_the_oracle_finite():
    rng = np.random.default_rng(3)
    w = World()
    ids = scenes.random_mix(16, seed=4).build(w)
    o = oracle_from_world(w, DT)
    for _ in range(10):
        o.edit_bodies(*random_edits(rng, ids, 12))
        o.step(DT)
        s = o.states()
        assert np.isfinite(s["position"]).all() and np.isfinite(s["velocity"]).all()
    o.close()
    w.close()


def test_the_boundary_refuses_unknown_bodies_and_kinds():
    w = World()
    scenes.sphere_row(2).build(w)
    with pytest.raises(DynamisError):
        w.edit_bodies([7], R.body_edit(R.EDIT_FORCE, force=(1.0, 0.0, 0.0)))
    with pytest.raises(DynamisError):
        w.edit_bodies([0], R.body_edit(9))
    with pytest.raises(ValueError):
        w.edit_bodies([0, 1], R.body_edit(R.EDIT_WAKE))
    w.edit_bodies([], np.zeros(0, R.BODY_EDIT))
    w.apply_impulse(1, (0.0, 1.0, 0.0))
    w.close()


def test_the_record_layout_matches_the_abi():
    assert R.BODY_EDIT.itemsize == 160 and R.BODY_EDIT.fields["state"][1] == 16
