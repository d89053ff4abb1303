# SPDX-License-Identifier: MIT
"""CPU checks of the oracle and of the product's host-side logic (no GPU).

- The oracle's AVBD math passes the reference's own 105-fixture suite
  (tests/solver/geometry_constraint_cases.hpp) when built against it.
- The oracle matches the committed golden vectors produced by the
  reference's C++ mirror of constraint_math.slang (rel 2e-5 / abs 2e-6,
  the reference validator's default tolerance).
- Mesh preparation of the product library equals the oracle's bit for bit.
- The oracle's broadphase equals brute-force pair enumeration; its colouring
  has the greedy first-fit property; a pyramid stays standing; FP32 and the
  FP64 replay stay close over the first frames.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from pmb200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF = os.environ.get("PMB_REFERENCE_ROOT", "/root/reference")


def _num(v):
    if isinstance(v, str):
        return {"nan": np.nan, "inf": np.inf, "-inf": -np.inf}[v]
    return v


def _arr(rows):
    return np.array([[_num(x) for x in r] for r in rows], np.float32)


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "avbd_core_vectors.json")) as f:
        return json.load(f)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "tests", "solver")), reason="reference checkout absent")
def test_reference_fixture_suite_passes_on_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "pin", f"REF={REF}"], check=True)
    out = subprocess.run([os.path.join(REPO, "oracle", "_ref", "pin_reference_fixtures")], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "oracle fixtures: 85/85 passed" in out.stdout


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "tests", "solver")), reason="reference checkout absent")
def test_reference_spatial_fixtures_pass_on_oracle():
    """The oracle's broadphase pair predicate on the reference's spatial
    fixtures (rigid_spatial_tests.cpp's shared-query scenario, the leaves and
    queries of spatial_build_primitives_tests.cpp), compiled against the
    reference's spatial headers."""
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "pin", f"REF={REF}"], check=True)
    out = subprocess.run([os.path.join(REPO, "oracle", "_ref", "pin_spatial_fixtures")], capture_output=True,
                         text=True)
    assert out.returncode == 0, out.stdout[-2000:]
    assert "spatial pins: passed" in out.stdout


def test_block_solve_golden(golden):
    n_ok = 0
    for b in golden["blocks"]:
        h = np.array([_num(x) for x in b["h"]], np.float32)
        g = np.array([_num(x) for x in b["g"]], np.float32)
        ok, d = O.block_solve(h, g)
        assert ok == bool(b["solved"])
        if ok:
            ref = np.array([_num(x) for x in b["delta"]], np.float64)
            n_ok += np.allclose(d, ref, rtol=2e-5, atol=2e-6)
    # A few high-condition fixtures are validated by backward error in the
    # reference; componentwise agreement holds for the rest.
    assert n_ok >= 0.97 * sum(b["solved"] for b in golden["blocks"])


def test_dual_contact_row_golden(golden):
    for e in golden["duals"]:
        v = [_num(x) for x in e["in"]]
        w = O.warm_start(v[0], v[1], v[6])
        u = O.update_dual(*v[:7])
        got = np.array([w[0], w[1], u[2], u[0], u[1]], np.float32)
        np.testing.assert_allclose(got, np.array([_num(x) for x in e["out"]], np.float32), rtol=2e-5, atol=2e-6)
    for e in golden["contacts"]:
        v = [_num(x) for x in e["in"]]
        got = O.project_contact(v[:3], v[3])
        np.testing.assert_allclose(got, np.array([_num(x) for x in e["out"]], np.float32), rtol=2e-5, atol=2e-6)
    for e in golden["rows"]:
        got = O.row_eval(np.array([_num(x) for x in e["in"]], np.float32))
        np.testing.assert_allclose(got, np.array([_num(x) for x in e["out"]], np.float32), rtol=2e-5, atol=2e-6)


def _meshes():
    yield scenes.box_mesh((0.5, 0.5, 0.5))
    yield scenes.box_mesh((0.31, 0.72, 1.4))
    v, t = scenes.capsule_mesh(0.05, 0.4)
    yield v, scenes._fix_winding(v, t)
    # An open (non-closed) mesh: one quad.
    yield np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32), np.array([0, 1, 2, 0, 2, 3], np.uint32)


def test_mesh_preparation_matches_oracle():
    pytest.importorskip("pmb200.core")
    from pmb200 import core
    if not os.path.exists(core.LIB_PATH):
        pytest.skip("core library not built")
    for v, t in _meshes():
        a = O.prepare_mesh(v, t)
        b = core.prepare_mesh(v, t)
        assert a[0] == b[0]
        assert np.array_equal(a[1], b[1])
        if a[0]:
            assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))
        assert np.array_equal(a[3].view(np.uint32), b[3].view(np.uint32))


def test_box_and_capsule_take_the_convex_face_path():
    for v, t in list(_meshes())[:3]:
        convex, idx, planes, _ = O.prepare_mesh(v, t)
        assert convex and len(idx) <= 96
        assert np.allclose(np.linalg.norm(planes[:, :3], axis=1), 1.0, atol=1e-6)


def _brute_pairs(lo, hi, motion, n):
    out = []
    for a in range(n):
        if motion[a] != scenes.DYNAMIC:
            continue
        for b in range(n):
            if b == a:
                continue
            if motion[b] == scenes.DYNAMIC and not a < b:
                continue
            if np.all(hi[b] >= lo[a]) and np.all(hi[a] >= lo[b]):
                out.append(a * n + b)
    return np.array(out, np.uint32)


def test_broadphase_equals_brute_force():
    s = scenes.box_pile((5, 4, 5), seed=3, spacing=1.5)
    w = O.OracleWorld(s)
    for _ in range(25):
        w.step()
        lo, hi = w.aabbs()
        pairs = w.candidate_pairs()
        assert np.array_equal(pairs, _brute_pairs(lo, hi, s.bodies["motion"], s.n))


def test_colouring_is_first_fit_in_index_order():
    s = scenes.box_pile((5, 4, 5), seed=5, spacing=1.5)
    w = O.OracleWorld(s)
    for _ in range(40):
        w.step()
    colors, parents = w.graph()
    codes, counts, _ = w.manifolds()
    n = s.n
    dyn = s.bodies["motion"] == scenes.DYNAMIC
    nbr = {i: set() for i in range(n)}
    for c in codes:
        a, b = int(c // n), int(c % n)
        if dyn[a] and dyn[b]:
            nbr[a].add(b)
            nbr[b].add(a)
    for v in range(n):
        if not dyn[v]:
            continue
        lower = {int(colors[u]) for u in nbr[v] if u < v}
        mex = 0
        while mex in lower:
            mex += 1
        assert colors[v] == mex
        # island roots are the lowest index of each connected component
        assert parents[v] <= v and parents[parents[v]] == parents[v]


def test_pyramid_stays_standing():
    s = scenes.pyramid()
    w = O.OracleWorld(s)
    x0 = s.states["x"].copy()
    for _ in range(120):
        st = w.step()
        assert st["status"] == 0
    x = w.states()["x"]
    drift = np.abs(x[1:] - x0[1:]).max()
    assert drift < 0.02, drift
    codes, counts, contacts = w.manifolds()
    pen = max(contacts[k, :counts[k], 6].max() for k in range(len(codes)))
    assert pen < 5e-3


def test_fp32_tracks_fp64_replay():
    s = scenes.pyramid()
    a = O.OracleWorld(s)
    b = O.OracleWorld(s, fp64=True)
    for f in range(30):
        a.step()
        b.step()
    xa, xb = a.states(), b.states()
    assert np.abs(xa["x"] - xb["x"]).max() < 1e-3
    assert np.abs(xa["v"] - xb["v"]).max() < 1e-2


def test_chain_scene_shapes():
    s = scenes.chains(count=4, links=8)
    assert s.n == 4 * (8 + 2)
    assert len(s.joints) == 4 * 9
    w = O.OracleWorld(s)
    for _ in range(10):
        st = w.step()
    flags, applied, counts = w.joints()
    assert (counts == 3).all() and (flags & 1).all()
    assert np.isfinite(w.states()["x"]).all()


def test_scene_batch_concatenates_independent_scenes():
    parts = [scenes.pyramid(levels=3), scenes.chains(count=2, links=3), scenes.box_pile((2, 2, 2), seed=1)]
    b = scenes.batch(parts)
    assert b.n == sum(p.n for p in parts)
    assert list(np.bincount(b.body_scene)) == [p.n for p in parts]
    assert list(b.scene_iterations) == [p.iterations for p in parts]
    assert len(b.mesh_vertex_offsets) - 1 == sum(len(p.mesh_vertex_offsets) - 1 for p in parts)
    # joints stay inside their scene
    sa, sb = b.body_scene[b.joints["body_a"]], b.body_scene[b.joints["body_b"]]
    assert np.array_equal(sa, sb) and (sa == 1).all()
    # body k of part 1 keeps its mesh geometry
    off = parts[0].n
    m = b.bodies["mesh"][off]
    m0 = parts[1].bodies["mesh"][0]
    v = b.vertices[b.mesh_vertex_offsets[m]:b.mesh_vertex_offsets[m + 1]]
    v0 = parts[1].vertices[parts[1].mesh_vertex_offsets[m0]:parts[1].mesh_vertex_offsets[m0 + 1]]
    assert np.array_equal(v, v0)


def test_joint_zoo_runs_every_joint_type():
    """Every joint type steps without non-finite state; the under-rated
    point joints break, all others stay enabled and keep their rows."""
    z = scenes.joint_zoo()
    kinds = sorted(set(int(t) for t in z.joints["type"]))
    assert kinds == list(range(8))
    o = O.OracleWorld(z)
    for _ in range(30):
        st = o.step()
        assert st["status"] == 0
    x = o.states()
    assert np.isfinite(x["x"]).all() and np.isfinite(x["q"]).all()
    flags, applied, counts = o.joints()
    breakable = z.joints["breaking_threshold"] > 0
    assert (flags[breakable] & 2).all() and (counts[breakable] == 0).all()
    assert (flags[~breakable] == 1).all() and (counts[~breakable] > 0).all()


def test_fixed_collision_groups_filter_candidates():
    """Bodies joined by collision-disabling fixed joints share a collision
    group (pm_build_fixed_collision_groups, geometry.slang:3102-3136) and no
    pair inside a group is a candidate (:902-904): A-C of the welded bars and
    D-E (joined through a static post) stay out, the outsider resting on C
    stays in. Letting the B-C weld collide splits the bars' group."""
    for disable_bc in (True, False):
        s = scenes.welded_groups(disable_bc=disable_bc)
        o = O.OracleWorld(s)
        assert o.step()["status"] == 0
        pairs = {(int(c) // s.n, int(c) % s.n) for c in o.candidate_pairs()}
        assert ((1, 3) in pairs) == (not disable_bc)
        assert ((2, 3) in pairs) == (not disable_bc)
        assert (1, 2) not in pairs and (5, 6) not in pairs
        assert (3, 7) in pairs
    o = O.OracleWorld(scenes.welded_groups())
    for _ in range(60):
        assert o.step()["status"] == 0
    x = o.states()["x"]
    # the welded bars settle on the ground where they were put
    assert np.allclose(x[1:4, 0], [-1.0, -0.5, 0.0], atol=1e-3) and np.allclose(x[1:4, 1], 0.101, atol=2e-3)


def test_triangle_mesh_path_holds_concave_and_large_meshes():
    """Pairs the convex face path does not take go to the triangle-mesh path
    (geometry.slang:2156-2299, :1359-1584): boxes dropped into a concave
    trough come to rest on its floor between its walls, a concave L rests on
    the ground with another on top of it, a 64-triangle capsule lies on the
    ground on one of its faces."""
    s = scenes.mesh_mix()
    o = O.OracleWorld(s)
    for _ in range(150):
        st = o.step()
        assert st["status"] == 0
    x = o.states()["x"]
    assert np.isfinite(x).all()
    floor = 0.2 + 0.15
    assert np.all(np.abs(x[2:5, 1] - floor) < 5e-3), x[2:5, 1]
    assert np.all(np.abs(x[2:5, 0]) < 0.8 - 0.15 + 1e-2)
    assert abs(x[5, 1] - 0.2) < 5e-3 and x[6, 1] > 0.1
    assert abs(x[7, 1] - 0.2 * np.cos(np.pi / 16)) < 5e-3
    # every pair with contacts has at most eight, and the trough's floor
    # carries the three boxes
    codes, counts, _ = o.manifolds()
    assert counts.max() <= 8
    pairs = {(int(c) // s.n, int(c) % s.n) for c in codes}
    assert {(2, 1), (3, 1), (4, 1)} <= pairs
    # With 5 mm margins the first box falls 4.7 cm per tick onto the trough
    # floor: only the swept triangle ranges (:1921-2155) stop it there.
    o = O.OracleWorld(scenes.mesh_mix(margin=0.005))
    for _ in range(150):
        assert o.step()["status"] == 0
    assert abs(o.states()["x"][2, 1] - floor) < 5e-3


@pytest.mark.parametrize("kind", [scenes.PISTON, scenes.SLIDER])
def test_guided_contacts_stop_a_piston_at_the_guided_offset(kind):
    """A box on an unbreakable piston (slider) joint to a static anchor slides
    at 3 m/s into a static stop: the pair is guided (geometry.slang:373-377),
    so the face path skips it and the swept triangle ranges give contacts
    merged by guide direction (:1129-1170) -- one contact for the whole face
    -- and the box rests within the guided offset (1e-4 m) of the stop."""
    s = scenes.guided_stop(kind)
    o = O.OracleWorld(s)
    counts = []
    for _ in range(40):
        st = o.step()
        assert st["status"] == 0
        counts.append(int(st["contacts"]))
    x = o.states()
    stop_face = 2.0 - 0.2 - 0.2
    assert stop_face - 2e-4 <= x["x"][1, 0] <= stop_face
    assert abs(x["v"][1, 0]) < 1e-3
    assert max(counts) == 1 and sum(counts) >= 3


def test_fp32_arctangent_and_cotangent_accuracy():
    """The FP32 tick's own atan2 (first quadrant) and x cot(x) on [0, pi/2]
    (addition formula plus Maclaurin series, basic operations only): within
    3 ulp of the float64 atan2, and 3e-7 absolute of x cos(x) / sin(x)."""
    rng = np.random.Generator(np.random.Philox(21))
    yx = rng.uniform(0.0, 1.0, (4000, 2)).astype(np.float32)
    yx[:200, 1] = 0.0                       # x = 0: pi/2
    yx[200:400, 0] = yx[200:400, 1]         # y = x: pi/4
    t = np.linspace(0.5, np.pi / 2, 4000).astype(np.float32)
    for (y, x), tt in zip(yx, t):
        a, c = O.trig_eval([y, x, tt])
        exact = np.arctan2(np.float64(y), np.float64(x))
        assert abs(float(a) - exact) <= 3 * float(np.spacing(np.float32(exact))), (y, x, a, exact)
        ref = np.float64(tt) * np.cos(np.float64(tt)) / np.sin(np.float64(tt))
        assert abs(float(c) - ref) <= 3e-7, (tt, c, ref)
