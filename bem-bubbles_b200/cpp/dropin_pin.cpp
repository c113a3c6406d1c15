// Drop-in Bem::ColocSimPin (Bem/Simulation/ColocSimPin.hpp in this directory): a bubble on the wall
// x = 0 with its contact line pinned to the wall.  The per-stage work -- assembly with the exchanged
// pinned columns, the solve, the velocities, the contact-line drift -- runs on the GPU through
// bem_set_pinned / bem_position_t_inout; the RK4 and Euler steps are LinLinSim's device steps, which
// honour the pins.  Remeshing is host-side mesh editing with the user's Bem/Mesh library; it keeps
// the new contact line on the old one (ColocSimPin.cpp:289-619).
#include <cmath>
#include <iostream>
#include <stdexcept>
#include <string>

#include "Bem/Simulation/ColocSimPin.hpp"
#include "Bem/Mesh/HalfedgeMesh.hpp"
#include "Bem/Mesh/MeshIO.hpp"
#include "Bem/Mesh/MeshManip.hpp"
#include "../../include/bem_b200.h"
#include "dropin_util.hpp"

namespace Bem {

using dropin::flat;
using dropin::unflat;

// The contact-angle drift law of the reference (ColocSimPin.cpp:126-136):
// v = beta (cos_eq - cos) + c_nl cos^3 / (cos^2 - 1), cos_eq = cos(130 deg).
static const real kDriftBeta = 0.2;
static const real kDriftCosEq = std::cos(130.0 / 180.0 * M_PI);
static const real kDriftNonlinear = 0.01;

void ColocSimPin::configure_context(bem_ctx* c) const {
    check(bem_set_pinned(c, (int64_t)N_pin, kDriftBeta, kDriftCosEq, kDriftNonlinear));
}

void ColocSimPin::assemble_matrices(Eigen::MatrixXd& G, Eigen::MatrixXd& H, Mesh const& m) const {
    bem_ctx* c = context(m);
    const Eigen::Index n = (Eigen::Index)m.verts.size();
    G.resize(n, n);
    H.resize(n, n);
    std::vector<double> x = flat(m.verts);
    check(bem_assemble(c, x.data(), G.data(), H.data()));
}

CoordVec ColocSimPin::position_t(Mesh const& m, PotVec& pot) const {
    bem_ctx* c = context(m);
    check(bem_set_V0(c, V_0));
    check(bem_set_psi(c, psi.data()));  // the stored psi stands in for pot at the pinned vertices
    std::vector<double> x = flat(m.verts), vel(3 * m.verts.size());
    check(bem_position_t_inout(c, x.data(), pot.data(), vel.data(), nullptr));
    return unflat(vel);
}

// ------------------------------------------------------------------ contact-line bookkeeping

// Moves the flagged vertices to the end of M.verts with the reference's scan (ColocSimPin.cpp:196-287):
// over the unsettled range [0, k), a flagged vertex trades places with vertex k-1, the range shrinks,
// and the vertex that came in is examined next.  `on_swap(i, j)` exchanges the caller's per-vertex
// data along.  The triangles are renumbered; returns the number of flagged vertices.
template <class Flagged, class OnSwap>
static size_t move_flagged_to_end(Mesh& M, Flagged flagged, OnSwap on_swap) {
    const size_t n = M.verts.size();
    std::vector<size_t> origin(n);  // origin[p] = old index of the vertex now at p
    for (size_t p = 0; p < n; ++p) origin[p] = p;
    size_t k = n, moved = 0;
    for (size_t i = 0; i < k;) {
        if (!flagged(i)) {
            ++i;
            continue;
        }
        std::swap(origin[i], origin[k - 1]);
        std::swap(M.verts[i], M.verts[k - 1]);
        on_swap(i, k - 1);
        --k;
        ++moved;
    }
    std::vector<size_t> where(n);
    for (size_t p = 0; p < n; ++p) where[origin[p]] = p;
    for (Triplet& t : M.trigs) {
        t.a = where[t.a];
        t.b = where[t.b];
        t.c = where[t.c];
    }
    return moved;
}

static const real kWallThreshold = 1e-5;  // |x| below which a vertex is on the wall

size_t ColocSimPin::set_x_boundary(Mesh& M, PotVec& phi_t, PotVec& psi_t) const {
    const size_t npin = move_flagged_to_end(
        M,
        [&](size_t i) {
            if (std::abs(M.verts[i].x) >= kWallThreshold) return false;
            M.verts[i].x = 0.0;
            return true;
        },
        [&](size_t i, size_t j) {
            std::swap(phi_t[i], phi_t[j]);
            std::swap(psi_t[i], psi_t[j]);
        });
    std::cout << "npin = " << npin << std::endl;
    return npin;
}

size_t ColocSimPin::set_x_boundary(Mesh& M) const {
    const size_t npin = move_flagged_to_end(
        M,
        [&](size_t i) {
            if (std::abs(M.verts[i].x) >= kWallThreshold) return false;
            M.verts[i].x = 0.0;
            return true;
        },
        [](size_t, size_t) {});
    std::cout << "npin = " << npin << std::endl;
    return npin;
}

void ColocSimPin::rearrange_boundary(Mesh& M, std::vector<bool> bound) const {
    move_flagged_to_end(
        M, [&](size_t i) { return (bool)bound[i]; },
        [&](size_t i, size_t j) {
            const bool t = bound[i];
            bound[i] = bound[j];
            bound[j] = t;
        });
}

// ------------------------------------------------------------------ remesh

// Vertex indices around the first boundary loop of a halfedge mesh, from bounds[0] along next.
static std::vector<size_t> boundary_loop(HalfedgeMesh const& he) {
    std::vector<size_t> loop;
    Halfedge* const start = he.bounds[0];
    Halfedge* h = start;
    do {
        loop.push_back(h->vert);
        h = h->next;
    } while (h != start);
    return loop;
}

// Offset (0-based, within the last `count` vertices of pts) of the vertex nearest to p; the first of
// equal distances wins.
static size_t nearest_in_tail(CoordVec const& pts, size_t count, vec3 const& p) {
    const size_t base = pts.size() - count;
    size_t best = 0;
    real dbest = (pts[base] - p).norm2();
    for (size_t j = 1; j < count; ++j) {
        const real d = (pts[base + j] - p).norm2();
        if (d < dbest) {
            dbest = d;
            best = j;
        }
    }
    return best;
}

// In-wall outward normal of the new contact line at each loop vertex: the mean of the wall-plane normals
// of its two loop edges, oriented along the vertex normal (ColocSimPin.cpp:436-489).  Indexed by the
// vertex's place among the last N_pin vertices of `ref` (the new mesh before relaxation).
static CoordVec contact_line_normals(HalfedgeMesh const& he, Mesh const& ref, size_t npin) {
    const std::vector<size_t> loop = boundary_loop(he);
    const std::vector<vec3> vnorm = generate_vertex_normals(he);
    const vec3 ex(1.0, 0.0, 0.0);
    const size_t n = loop.size();
    CoordVec out(npin);
    // the reference walks the loop starting at its third vertex; the order only shows in the log
    for (size_t s = 0; s < n; ++s) {
        const size_t k = (s + 2) % n;
        const vec3 prev = he.vpos[loop[(k + n - 1) % n]], here = he.vpos[loop[k]], next = he.vpos[loop[(k + 1) % n]];
        const size_t slot = nearest_in_tail(ref.verts, npin, here);
        vec3 wall = vnorm[loop[k]];
        const vec3 full = wall;
        wall.x = 0.0;
        wall.normalize();
        vec3 ea = (next - here).vec(ex), eb = (here - prev).vec(ex);
        ea.normalize();
        eb.normalize();
        vec3 nl = ea + eb;
        nl.normalize();
        if (nl.dot(full) < 0.0) nl = -nl;
        out[slot] = nl;
        const real dev = (nl - wall).norm();
        if (dev > 0.1) std::cout << "val = " << dev << ", nor = " << wall << ", nor_o = " << nl << std::endl;
    }
    return out;
}

// Where the ray p + s*d meets the old contact line (the closed polyline through the vertices `ring`
// of `old`): the segment hit with parameter t in [0, 1) and the smallest |s| (ColocSimPin.cpp:511-538).
struct LineHit {
    size_t seg;
    real s, t;
};
static LineHit hit_old_contact_line(Mesh const& old, std::vector<size_t> const& ring, vec3 const& p,
                                    vec3 const& d) {
    const size_t kp = ring.size();
    bool found = false;
    LineHit best{0, 0.0, 0.0};
    for (size_t j = 0; j < kp; ++j) {
        const vec3 edge = old.verts[ring[(j + 1) % kp]] - old.verts[ring[j]];
        const vec3 O = old.verts[ring[j]] - p;
        const real t = (O.vec(d)).x / (d.vec(edge)).x;
        const real s = d.dot(O + t * edge) / d.norm2();
        if (t >= 0.0 && t < 1.0 && (!found || std::abs(s) < std::abs(best.s))) {
            found = true;
            best = {j, s, t};
        }
    }
    if (!found) throw std::out_of_range("project_and_interpolate: no intersection at boundary");
    return best;
}

void ColocSimPin::remesh(real L) {
    std::cout << "begin remesh" << std::endl;
    test_negative();
    update_curvature_params();

    // the old contact line as indices of the current mesh, in loop order
    std::vector<size_t> old_ring;
    {
        HalfedgeMesh cur(mesh);
        for (size_t v : boundary_loop(cur))
            old_ring.push_back(mesh.verts.size() - N_pin + nearest_in_tail(mesh.verts, N_pin, cur.vpos[v]));
    }

    // topology edits: one split, collapses and flips (ColocSimPin.cpp:349-372)
    HalfedgeMesh he(mesh);
    split_edges(he, curvature_params, L * 4.0 / 3.0);
    collapse_edges(he, curvature_params, L * 4.0 / 5.0);
    for (int pass = 0; pass < 2; ++pass) {
        flip_edges(he, 1);
        flip_edges(he, 1);
        collapse_edges(he, curvature_params, L * 4.0 / 5.0);
    }
    flip_edges(he, 1);
    flip_edges(he, 1);

    // the new contact line goes to the end of the vertex list
    Mesh next = generate_mesh(he);
    std::vector<bool> on_line(he.verts.size(), false);
    const std::vector<size_t> new_loop = boundary_loop(he);
    for (size_t v : new_loop) on_line[v] = true;
    rearrange_boundary(next, on_line);
    const Mesh before_relax = next;
    N_pin = new_loop.size();
    CoordVec normals = generate_vertex_normals(next);
    const CoordVec line_pts(next.verts.end() - (std::ptrdiff_t)N_pin, next.verts.end());

    // free vertices: relax, project back onto the old surface along the normals, interpolate phi and
    // psi, keep them off the wall (ColocSimPin.cpp:406-424)
    relax_vertices(next);
    next.verts.resize(next.verts.size() - N_pin);
    normals.resize(normals.size() - N_pin);
    std::vector<real> new_phi, new_psi;
    const CoordVec x0 = next.verts;
    const std::vector<real> old_phi = make_copy(phi), old_psi = make_copy(psi);
    dropin::project_interpolate(device_ctx(), next, normals, mesh, old_phi, new_phi, &old_psi, &new_psi, false);
    CoordVec shift = next.verts + (-1.0) * x0;
    next.verts = nopenetration(eps, 1.0, x0, shift);

    // contact-line vertices: cast along the in-wall normal onto the old contact line and interpolate
    // phi and psi on the segment hit (ColocSimPin.cpp:497-571); the rays and the hits are also written
    // as a diagnostic mesh with the old surface
    const CoordVec dirs = contact_line_normals(he, before_relax, N_pin);
    Mesh rays;
    PotVec ray_pots;
    const size_t kp = old_ring.size();
    for (size_t i = 0; i < N_pin; ++i) {
        vec3 p = line_pts[i];
        const vec3 d = dirs[i];
        const LineHit h = hit_old_contact_line(mesh, old_ring, p, d);
        const size_t ia = old_ring[h.seg], ib = old_ring[(h.seg + 1) % kp];
        const vec3 tail = p - d * 0.2;
        p += h.s * d;
        const size_t o = rays.verts.size();
        rays.verts.push_back(tail);
        rays.verts.push_back(mesh.verts[ia]);
        rays.verts.push_back(p);
        rays.verts.push_back(mesh.verts[ib]);
        rays.trigs.push_back(Triplet(o, o + 1, o + 2));
        rays.trigs.push_back(Triplet(o, o + 2, o + 3));
        const real phi_hit = (1.0 - h.t) * phi((Eigen::Index)ia) + h.t * phi((Eigen::Index)ib);
        const real psi_hit = (1.0 - h.t) * psi((Eigen::Index)ia) + h.t * psi((Eigen::Index)ib);
        ray_pots.push_back(0.0);
        ray_pots.push_back(phi((Eigen::Index)ia));
        ray_pots.push_back(phi_hit);
        ray_pots.push_back(phi((Eigen::Index)ib));
        next.verts.push_back(p);
        new_phi.push_back(phi_hit);
        new_psi.push_back(psi_hit);
    }
    rays.add(mesh);
    for (Eigen::Index i = 0; i < phi.size(); ++i) ray_pots.push_back(phi(i));
    export_ply_float("borderprojects/mesh-" + std::to_string(index++) + ".ply", rays, ray_pots);

    mesh = next;
    set_phi(new_phi);
    set_psi(new_psi);
    std::cout << "end_remesh" << std::endl;
    test_negative();
}

}  // namespace Bem
