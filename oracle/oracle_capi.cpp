// SPDX-License-Identifier: MIT
// ORACLE — test infrastructure only. C ABI over the CPU restatement so the
// Python tests, smoke() and bench.py's cpu_baseline leg can drive it. The
// product library never links or loads this file.
#include <cstring>
#include <cstdlib>
#include <memory>
#include <new>

#include "avbd_step.hpp"

using namespace oracle;

namespace {

struct Handle {
    bool fp64{};
    World<float> f;
    World<double> d;
};

template <class R>
void build(World<R>& w, uint32_t n, const BodyDesc* bodies, const StateDesc* states, uint32_t nm,
           const uint32_t* voff, const float* verts, const uint32_t* ioff, const uint32_t* idx, uint32_t nj,
           const JointDesc* joints) {
    w.n = n;
    w.body.assign(bodies, bodies + n);
    w.state.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        w.state[i] = to_state<R>(states[i]);
        w.state[i].q = qnormalize(w.state[i].q);
    }
    w.meshes.clear();
    for (uint32_t m = 0; m < nm; ++m)
        w.meshes.push_back(prepare_mesh<R>(verts + 3 * size_t(voff[m]), voff[m + 1] - voff[m], idx + ioff[m],
                                           ioff[m + 1] - ioff[m]));
    w.joints.resize(nj);
    for (uint32_t j = 0; j < nj; ++j) w.joints[j].d = joints[j];
    w.avbd.assign(n, AvbdBody<R>{});
    w.force.assign(n, {});
    w.torque.assign(n, {});
    w.impulse.assign(n, {});
    w.angular_impulse.assign(n, {});
    w.target.assign(n, State<R>{});
    w.target_set.assign(n, 0);
    w.saved.clear();
    w.epoch = 0;
}

template <class F> auto with(Handle* h, F&& fn) {
    return h->fp64 ? fn(h->d) : fn(h->f);
}

}  // namespace

extern "C" {

void* oracle_create(uint32_t n, const BodyDesc* bodies, const StateDesc* states, uint32_t nm, const uint32_t* voff,
                    const float* verts, const uint32_t* ioff, const uint32_t* idx, uint32_t nj,
                    const JointDesc* joints, int fp64) {
    Handle* h = new (std::nothrow) Handle;
    if (!h) return nullptr;
    h->fp64 = fp64 != 0;
    if (h->fp64)
        build(h->d, n, bodies, states, nm, voff, verts, ioff, idx, nj, joints);
    else
        build(h->f, n, bodies, states, nm, voff, verts, ioff, idx, nj, joints);
    return h;
}

void* oracle_clone(void* hp) {
    Handle* h = static_cast<Handle*>(hp);
    return new (std::nothrow) Handle(*h);
}

void oracle_destroy(void* h) { delete static_cast<Handle*>(h); }

int oracle_step(void* hp, const StepDesc* o, StepStats* out) {
    Handle* h = static_cast<Handle*>(hp);
    with(h, [&](auto& w) {
        step(w, *o);
        if (out) *out = w.stats;
        return 0;
    });
    return 0;
}

void oracle_get_states(void* hp, StateDesc* out) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        for (uint32_t i = 0; i < w.n; ++i) out[i] = from_state(w.state[i]);
        return 0;
    });
}

void oracle_set_states(void* hp, const StateDesc* in) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        using R = std::decay_t<decltype(w.state[0].x.x)>;
        for (uint32_t i = 0; i < w.n; ++i) w.state[i] = to_state<R>(in[i]);
        return 0;
    });
}

void oracle_apply_impulse(void* hp, uint32_t body, const float* linear, const float* angular) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        using R = std::decay_t<decltype(w.state[0].x.x)>;
        w.impulse[body] = add(w.impulse[body], v3<R>(linear));
        w.angular_impulse[body] = add(w.angular_impulse[body], v3<R>(angular));
        return 0;
    });
}

// Replace the pending inputs of the listed bodies (12 floats each: force,
// torque, linear impulse, angular impulse). runtime_rigid.cu.inc:265-294
// accumulates onto cleared accumulators; callers merge duplicates first.
void oracle_set_inputs(void* hp, uint32_t count, const uint32_t* bodies, const float* values) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        using R = std::decay_t<decltype(w.state[0].x.x)>;
        for (uint32_t k = 0; k < count; ++k) {
            const float* v = values + 12 * size_t(k);
            const uint32_t b = bodies[k];
            w.force[b] = v3<R>(v);
            w.torque[b] = v3<R>(v + 3);
            w.impulse[b] = v3<R>(v + 6);
            w.angular_impulse[b] = v3<R>(v + 9);
        }
        return 0;
    });
}

// runtime_rigid.cu.inc:197-230: target orientation normalised.
void oracle_set_targets(void* hp, uint32_t count, const uint32_t* bodies, const StateDesc* targets) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        using R = std::decay_t<decltype(w.state[0].x.x)>;
        for (uint32_t k = 0; k < count; ++k) {
            State<R> t = to_state<R>(targets[k]);
            t.q = qnormalize(t.q);
            w.target[bodies[k]] = t;
            w.target_set[bodies[k]] = 1;
        }
        return 0;
    });
}

// runtime_rigid.cu.inc:147-195: state replaced (orientation normalised),
// AvbdBody, accumulators and target cleared, rows of joints on the body reset.
void oracle_write_states(void* hp, uint32_t first, uint32_t count, const StateDesc* states) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        using R = std::decay_t<decltype(w.state[0].x.x)>;
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t b = first + k;
            State<R> s = to_state<R>(states[k]);
            s.q = qnormalize(s.q);
            w.state[b] = s;
            w.avbd[b] = AvbdBody<R>{};
            w.force[b] = w.torque[b] = w.impulse[b] = w.angular_impulse[b] = V3<R>{};
            w.target_set[b] = 0;
        }
        for (auto& j : w.joints) {
            const bool touches = (j.d.body_a >= first && j.d.body_a - first < count) ||
                                 (j.d.body_b >= first && j.d.body_b - first < count);
            if (touches)
                for (auto& row : j.rows) row = Row<R>{};
        }
        return 0;
    });
}

uint32_t oracle_candidate_pairs(void* hp, uint64_t* out, uint32_t cap) {
    return with(static_cast<Handle*>(hp), [&](auto& w) {
        uint32_t n = uint32_t(w.candidate_pairs.size());
        for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = w.candidate_pairs[i];
        return n;
    });
}

// Per active (non-empty) pair: code, count; per contact: normal[3], point[3],
// penetration, error[3], dual lambda/penalty x3, anchors a/b -> 22 floats.
uint32_t oracle_manifolds(void* hp, uint64_t* codes, uint32_t* counts, float* contacts, uint32_t cap) {
    return with(static_cast<Handle*>(hp), [&](auto& w) {
        uint32_t n = uint32_t(w.active_pairs.size());
        if (cap < n) return n;
        for (uint32_t k = 0; k < n; ++k) {
            codes[k] = w.active_pairs[k];
            counts[k] = w.manifolds[k].count;
            for (uint32_t p = 0; p < 8; ++p) {
                float* o = contacts + (size_t(k) * 8 + p) * 22;
                const auto& c = w.manifolds[k].c[p];
                float v[22] = {float(c.normal.x), float(c.normal.y), float(c.normal.z), float(c.point.x),
                               float(c.point.y), float(c.point.z), float(c.penetration), float(c.error.x),
                               float(c.error.y), float(c.error.z), float(c.dual[0].lambda), float(c.dual[0].penalty),
                               float(c.dual[1].lambda), float(c.dual[1].penalty), float(c.dual[2].lambda),
                               float(c.dual[2].penalty), float(c.anchor_a.x), float(c.anchor_a.y),
                               float(c.anchor_a.z), float(c.anchor_b.x), float(c.anchor_b.y), float(c.anchor_b.z)};
                for (int q = 0; q < 22; ++q) o[q] = v[q];
            }
        }
        return n;
    });
}

// Contact events of the latest tick as the reference writes them
// (pm_prepare_parallel_contact_events, geometry.slang:2902-2939: every point
// of every active pair in order, up to the capacity, penetration clamped at
// 0; impulses from pm_save_rigid_contact_cache, :3028-3043: accumulated for
// persistent contacts, else the reported ones). 13 words per event: body,
// collider (as float bit patterns of uint32), position, normal,
// penetration, normal impulse, friction impulse. Returns the event count.
uint32_t oracle_contact_events(void* hp, float* out, uint32_t capacity) {
    return with(static_cast<Handle*>(hp), [&](auto& w) {
        uint32_t cursor = 0;
        const uint32_t n = w.n;
        for (uint32_t k = 0; k < w.active_pairs.size(); ++k) {
            const auto& m = w.manifolds[k];
            const uint32_t a = uint32_t(w.active_pairs[k] / n), b = uint32_t(w.active_pairs[k] % n);
            for (uint32_t p = 0; p < m.count; ++p, ++cursor) {
                if (cursor >= capacity || !out) continue;
                const auto& c = m.c[p];
                float* o = out + size_t(cursor) * 13;
                std::memcpy(&o[0], &a, 4);
                std::memcpy(&o[1], &b, 4);
                const float v[11] = {float(c.point.x), float(c.point.y), float(c.point.z), float(c.normal.x),
                                     float(c.normal.y), float(c.normal.z),
                                     float(c.penetration > 0 ? c.penetration : 0),
                                     float(c.persistent ? c.acc_n : c.rep_n),
                                     float(c.persistent ? c.acc_f.x : c.rep_f.x),
                                     float(c.persistent ? c.acc_f.y : c.rep_f.y),
                                     float(c.persistent ? c.acc_f.z : c.rep_f.z)};
                for (int q = 0; q < 11; ++q) o[2 + q] = v[q];
            }
        }
        return cursor < capacity ? cursor : capacity;
    });
}

void oracle_graph(void* hp, uint32_t* colors, uint32_t* parents) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        for (uint32_t i = 0; i < w.n; ++i) {
            if (colors) colors[i] = w.avbd[i].color;
            if (parents) parents[i] = w.avbd[i].parent;
        }
        return 0;
    });
}

uint32_t oracle_residual_trace(void* hp, float* out, uint32_t cap) {
    return with(static_cast<Handle*>(hp), [&](auto& w) {
        uint32_t n = uint32_t(w.residual_trace.size());
        for (uint32_t i = 0; i < n && i < cap; ++i) out[i] = float(w.residual_trace[i]);
        return n;
    });
}

void oracle_aabbs(void* hp, float* lo, float* hi) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        for (uint32_t i = 0; i < w.n; ++i) {
            lo[3 * i] = float(w.aabb_lo[i].x);
            lo[3 * i + 1] = float(w.aabb_lo[i].y);
            lo[3 * i + 2] = float(w.aabb_lo[i].z);
            hi[3 * i] = float(w.aabb_hi[i].x);
            hi[3 * i + 1] = float(w.aabb_hi[i].y);
            hi[3 * i + 2] = float(w.aabb_hi[i].z);
        }
        return 0;
    });
}

// Joint state after the last tick: enabled, broken, applied impulse, rows.
void oracle_joints(void* hp, uint32_t* flags, float* applied, uint32_t* counts) {
    with(static_cast<Handle*>(hp), [&](auto& w) {
        for (size_t j = 0; j < w.joints.size(); ++j) {
            flags[j] = w.joints[j].enabled | (w.joints[j].broken << 1);
            applied[j] = float(w.joints[j].applied);
            counts[j] = w.joints[j].count;
        }
        return 0;
    });
}

// Mesh preparation: reordered indices, per-triangle planes (n, d), bounds.
int oracle_prepare_mesh(const float* verts, uint32_t nv, const uint32_t* idx, uint32_t ni, uint32_t* out_idx,
                        float* out_planes, float* out_bounds) {
    Mesh<float> m = prepare_mesh<float>(verts, nv, idx, ni);
    for (uint32_t i = 0; i < ni; ++i) out_idx[i] = m.idx[i];
    for (size_t t = 0; t < m.planes.size(); ++t) {
        out_planes[4 * t] = m.planes[t].n.x;
        out_planes[4 * t + 1] = m.planes[t].n.y;
        out_planes[4 * t + 2] = m.planes[t].n.z;
        out_planes[4 * t + 3] = m.planes[t].d;
    }
    float b[10] = {m.lo.x, m.lo.y, m.lo.z, m.hi.x, m.hi.y, m.hi.z, m.center.x, m.center.y, m.center.z, m.radius};
    for (int i = 0; i < 10; ++i) out_bounds[i] = b[i];
    return m.convex ? 1 : 0;
}

// ---- core math entry points for the golden vectors
int oracle_block_solve(const float* h21, const float* g6, float* out6) {
    Block<float> b{};
    for (int i = 0; i < 21; ++i) b.h[i] = h21[i];
    for (int i = 0; i < 6; ++i) b.g[i] = g6[i];
    Vec6<float> d{};
    bool ok = block_solve(b, d);
    for (int i = 0; i < 6; ++i) out6[i] = d.v[i];
    return ok ? 1 : 0;
}
void oracle_warm_start(float lambda, float penalty, float stiffness, float* out2) {
    Dual<float> d = warm_start(Dual<float>{lambda, penalty}, stiffness);
    out2[0] = d.lambda;
    out2[1] = d.penalty;
}
void oracle_update_dual(float lambda, float penalty, float error, float beta, float lo, float hi, float stiffness,
                        float* out3) {
    Dual<float> d{lambda, penalty};
    Dual<float> u = update_dual(d, error, beta, lo, hi, stiffness);
    out3[0] = u.lambda;
    out3[1] = u.penalty;
    out3[2] = dual_force(d, error, lo, hi);
}
void oracle_project_contact(const float* trial3, float friction, float* out6) {
    Force3<float> t{trial3[0], trial3[1], trial3[2]};
    Force3<float> p = project_contact(t, friction), s = stiffness_scales(t, friction);
    out6[0] = p.n;
    out6[1] = p.t0;
    out6[2] = p.t1;
    out6[3] = s.n;
    out6[4] = s.t0;
    out6[5] = s.t1;
}
// values: a[6] b[6] lambda penalty error velocity lower upper stiffness
// damping beta reference_force, da[6] db[6] dt diag[6] first -> out: error,
// The FP32 arctangent and x cot(x) the oracle's tick uses: in (y, x, t),
// out (atan2(y, x), t cos(t) / sin(t)).
void oracle_trig_eval(const float* v, float* out2) {
    out2[0] = atan2_q1(v[0], v[1]);
    out2[1] = x_cot(v[2]);
}

// trial, force, advanced lambda, advanced penalty, sum(g), sum(diag h)
void oracle_row_eval(const float* v, float* out7) {
    Row<float> r{};
    for (int i = 0; i < 6; ++i) { r.a.v[i] = v[i]; r.b.v[i] = v[6 + i]; }
    r.dual = {v[12], v[13]};
    r.error = v[14];
    r.velocity = v[15];
    r.lower = v[16];
    r.upper = v[17];
    r.stiffness = v[18];
    r.damping = v[19];
    r.beta = v[20];
    r.reference_force = v[21];
    Vec6<float> a{}, b{};
    for (int i = 0; i < 6; ++i) { a.v[i] = v[22 + i]; b.v[i] = v[28 + i]; }
    float dt = v[34];
    Block<float> blk{};
    for (int i = 0; i < 6; ++i) blk.h[bidx(i, i)] = v[35 + i];
    row_accumulate(blk, r, v[41] != 0.0f, a, b, dt);
    Row<float> adv = row_advance(r, a, b);
    out7[0] = row_error(r, a, b);
    out7[1] = row_trial(r, a, b, dt);
    out7[2] = row_force(r, a, b, dt);
    out7[3] = adv.dual.lambda;
    out7[4] = adv.dual.penalty;
    float gs = 0, ds = 0;
    for (int i = 0; i < 6; ++i) { gs += blk.g[i]; ds += blk.h[bidx(i, i)]; }
    out7[5] = gs;
    out7[6] = ds;
}

}  // extern "C"
