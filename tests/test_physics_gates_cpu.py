# SPDX-License-Identifier: MIT
"""The physical-gate measures on known geometry, and the gates on the CPU
oracle's own trajectory of the 55-cube pyramid (the checker's physics must
pass the bounds the GPU runs are held to)."""
import numpy as np

from pmb200 import scenes
import oracle as O
import physics_gates as G

I = np.array([[0.0, 0.0, 0.0, 1.0]])


def test_box_overlap_known_cases():
    h = np.array([[0.5, 0.5, 0.5]])
    # face to face, 0.1 m overlap; 0.2 m apart; edge-on after a 45 degree turn
    assert np.isclose(G.box_overlap([[0, 0, 0]], I, h, [[0.9, 0, 0]], I, h, )[0], 0.1)
    assert np.isclose(G.box_overlap([[0, 0, 0]], I, h, [[1.2, 0, 0]], I, h)[0], -0.2)
    s = np.sin(np.pi / 8)
    q45 = np.array([[0.0, s, 0.0, np.cos(np.pi / 8)]])
    d = G.box_overlap([[0, 0, 0]], I, h, [[1.2, 0, 0]], q45, h)[0]
    assert np.isclose(d, 0.5 + np.sqrt(0.5) - 1.2)
    # a thin ground slab under a cube resting 1 mm into it
    g = np.array([[20.0, 0.5, 20.0]])
    assert np.isclose(G.box_overlap([[0, -0.5, 0]], I, g, [[3, 0.499, 1]], I, h)[0], 0.001)


def test_segment_distance_and_energy():
    p0, p1 = np.array([[0.0, 0, 0]]), np.array([[1.0, 0, 0]])
    q0, q1 = np.array([[0.5, 1, -1]]), np.array([[0.5, 1, 1]])
    assert np.isclose(G.segment_distance(p0, p1, q0, q1)[0], 1.0)
    s = scenes.pyramid(levels=2)
    st = s.states.copy()
    st["v"][:] = 0
    st["w"][:] = 0
    dyn = s.bodies["motion"] == scenes.DYNAMIC
    m = 1.0 / s.bodies["inv_mass"][dyn].astype(np.float64)
    assert np.isclose(G.energy(s, st), np.sum(m * 9.81 * st["x"][dyn, 1]))


def test_oracle_pyramid_meets_the_stack_gates():
    """120 ticks to settle, then 240 settled ticks of the legacy pyramid on
    the oracle: penetration <= 5 mm, settled drift <= 1 cm, rotation drift
    <= 0.035 rad, energy growth <= 5 %, no tunnelling."""
    s = scenes.pyramid()
    w = O.OracleWorld(s)
    dyn = s.bodies["motion"] == scenes.DYNAMIC
    pen, rot, tunnel = 0.0, 0.0, 0
    ys, energies = [], []
    for tick in range(360):
        w.step()
        st = w.states()
        codes, _, _ = w.manifolds()
        pairs = np.stack([codes.astype(np.int64) // s.n, codes.astype(np.int64) % s.n], axis=1)
        pen = max(pen, G.pair_penetration(s, st, pairs))
        rot = max(rot, float(G.rotation_angle(st["q"][dyn]).max()))
        tunnel += int((st["x"][dyn, 1] < 0.0).sum())
        if tick >= 120:
            ys.append(st["x"][dyn, 1].copy())
            energies.append(G.energy(s, st))
    drift = float((np.max(ys, axis=0) - np.min(ys, axis=0)).max())
    growth = max(energies) / energies[0] - 1.0
    print(f"oracle pyramid: penetration {pen:.3g} m, drift {drift:.3g} m, rotation {rot:.3g} rad, "
          f"energy growth {growth:.3g}, tunnelling {tunnel}")
    assert pen <= 0.005 and drift <= 0.01 and rot <= 0.035 and growth <= 0.05 and tunnel == 0


def test_convex_overlap_matches_box_overlap_and_capsules():
    """The general convex-mesh measure equals the oriented-box one on boxes,
    and two tessellated capsules side by side overlap by the distance their
    flat faces cross."""
    rng = np.random.Generator(np.random.Philox(5))
    s = scenes.box_pile((3, 2, 3), seed=3, spacing=0.9)
    st = s.states.copy()
    q = rng.normal(size=(s.n, 4))
    st["q"] = q / np.linalg.norm(q, axis=1, keepdims=True)
    dyn = np.flatnonzero(s.bodies["motion"] == scenes.DYNAMIC)
    a, b = dyn[:-1], dyn[1:]
    half = G.mesh_half_extents(s)
    ref = G.box_overlap(st["x"][a], st["q"][a], half[a], st["x"][b], st["q"][b], half[b])
    assert (ref > 0).sum() >= 3   # some of these spawn neighbours interpenetrate
    for k in range(len(a)):
        got = G.convex_overlap(s, st, a[k:k + 1], b[k:k + 1])[0]
        # Penetration depths agree; for separated pairs the mesh's triangle
        # diagonals only add axes that separate further (both negative).
        assert np.isclose(max(got, 0.0), max(ref[k], 0.0), atol=1e-9), (k, got, ref[k])
    c = scenes.chains(count=2, links=1, spacing=0.09)
    cs = c.states.copy()
    links = np.flatnonzero(c.bodies["mesh"] == c.bodies["mesh"][1])[:2]
    d = cs["x"][links[1], 0] - cs["x"][links[0], 0]
    got = G.convex_overlap(c, cs, links[:1], links[1:2])[0]
    # hexagon rings of radius 0.05 with a vertex on the x axis: the smallest
    # separating translation is along a side face's normal (30 degrees off
    # x), where each link reaches r cos 30 and the centres are d cos 30 apart
    assert np.isclose(got, (0.1 - abs(d)) * np.cos(np.pi / 6), atol=1e-6), (got, d)
