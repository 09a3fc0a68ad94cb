// dem_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU, FP64, single-threaded restatement of MercuryDPM's DEM time step for
// the paths the GPU engine implements. It is the checker the parity tests
// compare the CUDA path against; nothing in the product links or calls it.
// It is itself pinned against the reference build in oracle/_ref and the
// reference's own known-answer tests (tests/test_oracle.py).
//
// Step order follows DPMBase::computeOneTimeStep (Kernel/DPMBase.cc:4315-4389):
//   integrateBeforeForceComputation (BaseParticle.cc:718-752, then the walls:
//                                    BaseInteractable.cc:538-600)
//   checkInteractionWithBoundaries  (PeriodicBoundary.cc:374-395)
//   computeAllForces                (DPMBase.cc:3397-3526, :3113-3162, :3168-3215)
//   integrateAfterForceComputation  (BaseParticle.cc:760-776)
//   eraseOldInteractions            (InteractionHandler.cc:377-393)
// Periodic boundaries are restated with the reference's ghost semantics:
// a pair that meets across a boundary is evaluated twice, once from each real
// particle against the other's ghost (DPMBase.cc:3124-3127: ghost-ghost pairs
// are skipped, a real-ghost pair has the real particle as P because ghosts
// carry higher ids), and after the step the lower-index particle's view is
// kept while the other's view restarts from the reversed spring
// (InteractionHandler::removeObjectKeepingPeriodics, InteractionHandler.cc:316-368;
// BaseInteraction::copySwitchPointer, BaseInteraction.cc:340-356).
// The contact-law arithmetic is shared with the device code
// (mercurydpm_fork_b200/csrc/dem_laws.cuh), compiled here for the host.
//
// Insertion boundaries (InsertionBoundary::checkBoundaryBeforeTimeStep,
// Kernel/Boundaries/InsertionBoundary.cc:184-296) run after the periodic
// wrap and the deletions, before the forces, with the reference's random
// number generator restated here as the reference stores it (a vector of 607
// lags from which every draw drops the oldest), the placement of a
// CubeInsertionBoundary (CubeInsertionBoundary.cc:173-184) or
// ChuteInsertionBoundary (ChuteInsertionBoundary.cc:163-190), and the test of
// DPMBase::checkParticleForInteractionLocalPeriodic / ...Local
// (DPMBase.cc:4868-4958) against every particle, its copies made as the
// reference makes them. Input rows of radius 0 are free rows that placed
// particles fill in row order. Like the reference's HGrid lookup, the test
// does not see a particle that this step's drift shifted across a periodic
// boundary until a particle larger than any before has been placed (which
// rebuilds the reference's grid).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "../mercurydpm_fork_b200/csrc/dem_laws.cuh"
#include "../mercurydpm_fork_b200/csrc/dem_math.cuh"

using namespace dem;

namespace {

struct Particle {
    V3 x, v, w;
    Q4 q;
    double r, invm, invI;
    int species, id;
    bool fixed;
    bool deleted = false;
    bool wrapped = false; // the last periodic wrap moved it
    V3 F, T;
};

// RNG (Kernel/Math/RNG.cc): setRandomSeed fills the 607 lags from the linear
// congruential generator; getRandomNumber(lo, hi) appends
// fmod(lags[0] + lags[607 - 273], 1), drops lags[0] and returns lo + (hi - lo) x.
struct RefRng {
    std::vector<double> lags;
    explicit RefRng(unsigned long seed = 0)
    {
        const unsigned long a = 1103515245ul, c = 12345ul, m = 1024ul * 1024ul * 1024ul;
        unsigned long s = seed;
        for (int i = 0; i < 607; ++i) {
            s = (a * s + c) % m;
            lags.push_back(0.0 + 1.0 * (double)s / ((double)m + 1.0));
        }
    }
    double draw(double lo, double hi)
    {
        const double x = std::fmod(lags[0] + lags[607 - 273], 1.0);
        lags.erase(lags.begin());
        lags.push_back(x);
        const double range = hi - lo;
        return lo + range * x;
    }
};

// One insertion boundary and its state between steps.
struct InsBoundary {
    dem_insertion_boundary b;
    RefRng psd_rng;       // PSD::random_
    bool has_p0 = false;  // InsertionBoundary::p0
    double p0_r = 0.0;
    double volume = 0.0;  // volumeInserted_
    long long inserted = 0;
    // PSD::drawSample (Kernel/Math/PSD.cc:114-128)
    double draw_radius()
    {
        const double prob = psd_rng.draw(0, 1);
        const double* P = b.psd_probability;
        const int n = b.n_psd;
        const int high = (int)(std::lower_bound(P, P + n, prob) - P);
        const int low = std::max(0, high - 1);
        const double rMin = b.psd_radius[low], rMax = b.psd_radius[high];
        const double pMin = P[low], pMax = P[high];
        const double a = (prob - pMin) / (pMax - pMin);
        return a * rMin + (1 - a) * rMax;
    }
};

// Persistent interaction (InteractionHandler object). Key: (kind, P id, I id)
// kind 0: particle pair, P the lower id -- an ordinary pair, or the lower-id
//         particle's view of a periodic pair: after removeDuplicatePeriodicParticles
//         that view is the real-real interaction (InteractionHandler.cc:316-368),
//         so a pair that stops or starts being periodic keeps its spring;
// kind 1: the higher-id particle's view of a periodic pair (P real vs ghost of I);
// kind 2: wall (P particle, I wall index).
struct Inter {
    Springs s;
    unsigned stamp;
    unsigned eval;    // index of the last force evaluation that touched it
    double overlap;
    V3 force;
    double energy;
    bool periodic;
};

// One face of an IntersectionOfWalls: the InfiniteWall that
// IntersectionOfWalls::addObject(normal, point) creates (IntersectionOfWalls.cc:138-149).
struct Face {
    Q4 q;  // InfiniteWall orientation from the twice-normalised normal
    V3 p;  // point
    V3 n() const { return quat_axis(q); }
    double dist(V3 x) const { return quat_plane_distance(q, x, p); }
};

Q4 face_orientation(V3 n)
{
    // addObject's Vec3D::normalise, then Quaternion::setOrientationViaNormal
    // (Quaternion.cc:543-567), which normalises again
    for (int k = 0; k < 2; ++k) {
        const double l = sqrt(n.x * n.x + n.y * n.y + n.z * n.z);
        n = v3(n.x / l, n.y / l, n.z / l);
    }
    if (n.x <= -1 + 1e-14) return Q4{0, 0, 1, 0};
    const double h0 = 1.0 + n.x, h1 = 0.0 + n.y, h2 = 0.0 + n.z;
    const Q4 q{h0, 0.0, -h2, h1};
    const double l = sqrt(q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3);
    return Q4{q.q0 / l, q.q1 / l, q.q2 / l, q.q3 / l};
}

// Solution of the 3x3 system with rows r0, r1, r2 and right-hand side b by
// cofactors, in the term order of IntersectionOfWalls::setPointsAndLines
// (IntersectionOfWalls.cc:365-389, 399-433).
V3 cramer(V3 r0, V3 r1, V3 r2, double b0, double b1, double b2)
{
    const double c00 = r1.y * r2.z - r2.y * r1.z;
    const double c01 = r1.x * r2.z - r1.z * r2.x;
    const double c02 = r1.x * r2.y - r1.y * r2.x;
    const double inv = 1.0 / (+r0.x * c00 - r0.y * c01 + r0.z * c02);
    const double x = +c00 * b0 - (r0.y * r2.z - r0.z * r2.y) * b1 + (r0.y * r1.z - r0.z * r1.y) * b2;
    const double y = -c01 * b0 + (r0.x * r2.z - r0.z * r2.x) * b1 - (r0.x * r1.z - r1.x * r0.z) * b2;
    const double z = +(r1.x * r2.y - r2.x * r1.y) * b0 - (r0.x * r2.y - r2.x * r0.y) * b1 +
                     (r0.x * r1.y - r1.x * r0.y) * b2;
    return v3(x * inv, y * inv, z * inv);
}

struct Intersection {
    std::vector<Face> f;
    std::vector<V3> A, AB, C; // indexed as the reference's A_, AB_, C_

    void build(const dem_wall& w)
    {
        for (int n = 0; n < w.n_faces; ++n) {
            Face fc;
            fc.q = face_orientation(v3(w.faces[n][0], w.faces[n][1], w.faces[n][2]));
            fc.p = v3(w.faces[n][3], w.faces[n][4], w.faces[n][5]);
            f.push_back(fc);
            A.resize((size_t)(n + 1) * n / 2);
            AB.resize(A.size());
            for (int m = 0; m < n; ++m) {
                const V3 a = f[m].n(), b = f[n].n();
                V3 ab = v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
                const double l = sqrt(ab.x * ab.x + ab.y * ab.y + ab.z * ab.z);
                ab = v3(ab.x / l, ab.y / l, ab.z / l);
                const size_t id = (size_t)(n - 1) * n / 2 + m;
                AB[id] = ab;
                A[id] = cramer(b, a, ab, dot(f[n].p, b), dot(f[m].p, a), 0.0);
            }
            C.resize((size_t)(n + 1) * n * (n > 0 ? n - 1 : 0) / 6);
            for (int m = 0; m < n; ++m)
                for (int l = 0; l < m; ++l) {
                    const size_t id = (size_t)(n - 2) * (n - 1) * n / 6 + (size_t)(m - 1) * m / 2 + l;
                    C[id] = cramer(f[n].n(), f[m].n(), f[l].n(), dot(f[n].p, f[n].n()), dot(f[m].p, f[m].n()),
                                   dot(f[l].p, f[l].n()));
                }
        }
    }

    // IntersectionOfWalls::getDistanceAndNormal(const Vec3D&, ...) (IntersectionOfWalls.cc:567-712)
    bool distance(V3 x, double R, double& d, V3& nrm) const
    {
        if (f.empty()) return false;
        double d1 = -1e20, d2 = -1e20, d3 = -1e20;
        unsigned i1 = 0, i2 = 0, i3 = 0;
        for (unsigned i = 0; i < f.size(); ++i) {
            const double dc = f[i].dist(x);
            if (dc >= R) return false;
            if (dc > d1) {
                if (d1 > -R) {
                    if (d2 > -R) { d3 = d2; i3 = i2; }
                    d2 = d1; i2 = i1;
                }
                d1 = dc; i1 = i;
            } else if (dc < -R) {
                continue;
            } else if (dc > d2) {
                if (d2 > -R) { d3 = d2; i3 = i2; }
                d2 = dc; i2 = i;
            } else if (dc > d3) {
                d3 = dc; i3 = i;
            }
        }
        d = d1;
        if (d2 > -R) {
            const V3 D = x + f[i1].n() * d1;
            bool with2 = f[i2].dist(D) > 0.0;
            if (d3 > -R && f[i3].dist(D) > 0.0) {
                const V3 E = x + f[i2].n() * d2;
                const bool with3 = f[i3].dist(E) > 0.0;
                if (with2) {
                    if (with3) {
                        if (i2 > i3) std::swap(i2, i3);
                        auto tri = [](unsigned a) { return (a - 2) * (a - 1) * a / 6; };
                        auto pr = [](unsigned a) { return (a - 1) * a / 2; };
                        const unsigned idx = i1 < i2 ? tri(i3) + pr(i2) + i1
                                                     : (i1 < i3 ? tri(i3) + pr(i1) + i2 : tri(i1) + pr(i3) + i2);
                        nrm = x - C[idx];
                        d = sqrt(len2(nrm));
                        if (d <= R) { nrm = nrm / (-d); return true; }
                        if (d == d) return false;
                    }
                } else {
                    with2 = true;
                    d2 = d3;
                    i2 = i3;
                }
            }
            if (with2) {
                const unsigned idx = i1 > i2 ? (i1 - 1) * i1 / 2 + i2 : (i2 - 1) * i2 / 2 + i1;
                const V3 ac = x - A[idx];
                nrm = ac - AB[idx] * dot(ac, AB[idx]);
                d = sqrt(len2(nrm));
                if (d <= R) { nrm = nrm / (-d); return true; }
                if (d == d) return false;
            }
        }
        nrm = f[i1].n();
        return true;
    }
};

// Quaternion::rotate (back = false) / rotateBack (back = true), Quaternion.cc:570-640;
// the off-diagonal signs flip between the two (transpose)
V3 q_apply(Q4 q, V3 v, bool back)
{
    const double a = q.q0 * q.q0, b = q.q1 * q.q1, c = q.q2 * q.q2, e = q.q3 * q.q3;
    const double q01 = 2 * q.q0 * q.q1, q02 = 2 * q.q0 * q.q2, q03 = 2 * q.q0 * q.q3;
    const double q12 = 2 * q.q1 * q.q2, q13 = 2 * q.q1 * q.q3, q23 = 2 * q.q2 * q.q3;
    const double m01 = back ? q12 + q03 : q12 - q03, m02 = back ? q13 - q02 : q13 + q02;
    const double m10 = back ? q12 - q03 : q12 + q03, m12 = back ? q23 + q01 : q23 - q01;
    const double m20 = back ? q13 + q02 : q13 - q02, m21 = back ? q23 - q01 : q23 + q01;
    const double m00 = a + b - c - e, m11 = a - b + c - e, m22 = a - b - c + e;
    return v3(m00 * v.x + m01 * v.y + m02 * v.z, m10 * v.x + m11 * v.y + m12 * v.z, m20 * v.x + m21 * v.y + m22 * v.z);
}

struct Sim {
    dem_config cfg;
    dem_instance_desc inst;
    std::vector<dem_species_pair> species;
    std::vector<dem_wall> walls;
    std::vector<Intersection> wgeo;
    std::vector<Particle> p;
    std::map<std::tuple<int, int, int>, Inter> inter;
    unsigned nt = 0; // DPMBase::numberOfTimeSteps_
    unsigned evals = 0; // force evaluations so far
    double L[3], half[3];

    const dem_species_pair& sp(int a, int b) const
    {
        return species[inst.species_offset + a * inst.n_species + b];
    }

    void integrate_before()
    {
        const double dt = cfg.time_step;
        for (auto& q : p) {
            if (q.invm == 0.0) {
                q.x += q.v * dt;
                q.q = quat_rotate(q.q, q.w * dt);
            } else {
                q.v += ((q.F * q.invm) * 0.5) * dt;
                q.x += q.v * dt;
                if (cfg.rotation) {
                    const S33 I{q.invI, 0.0, 0.0, q.invI, 0.0, q.invI};
                    q.w += ((rotate_inverse_inertia(q.q, I) * q.T) * 0.5) * dt;
                    q.q = quat_rotate(q.q, q.w * dt);
                }
            }
        }
        for (auto& w : walls) { // BaseInteractable::integrateBeforeForceComputation: move, rotate
            const V3 dx = v3(w.velocity[0], w.velocity[1], w.velocity[2]) * dt;
            w.position[0] += dx.x; w.position[1] += dx.y; w.position[2] += dx.z;
            const Q4 q = quat_rotate(Q4{w.orientation[0], w.orientation[1], w.orientation[2], w.orientation[3]},
                                     v3(w.angular_velocity[0], w.angular_velocity[1], w.angular_velocity[2]) * dt);
            w.orientation[0] = q.q0; w.orientation[1] = q.q1; w.orientation[2] = q.q2; w.orientation[3] = q.q3;
        }
    }

    void integrate_after()
    {
        const double dt = cfg.time_step;
        for (auto& q : p) {
            if (q.invm == 0.0) continue;
            q.v += ((q.F * q.invm) * 0.5) * dt;
            if (cfg.rotation) {
                const S33 I{q.invI, 0.0, 0.0, q.invI, 0.0, q.invI};
                q.w += ((rotate_inverse_inertia(q.q, I) * q.T) * 0.5) * dt;
            }
        }
    }

    void wrap()
    {
        for (auto& q : p) q.wrapped = false;
        for (int k = 0; k < 3; ++k) {
            if (!((inst.periodic_mask >> k) & 1u)) continue;
            const double lo = inst.periodic_min[k], hi = inst.periodic_max[k];
            for (auto& q : p) {
                double* xc = &q.x.x;
                if (std::min(xc[k] - lo, hi - xc[k]) < 0) {
                    q.wrapped = true;
                    if (hi - xc[k] > xc[k] - lo)
                        xc[k] = xc[k] + L[k];
                    else
                        xc[k] = xc[k] - L[k];
                }
            }
        }
    }

    // One evaluation of DPMBase::computeInternalForce for P (real) against I
    // at position xi (I's real position or a ghost image).
    void pair(Particle& P, Particle& I, V3 xi, bool ghost)
    {
        const V3 branch = P.x - xi;
        const double d2 = len2(branch);
        const dem_species_pair& s = sp(P.species, I.species);
        const double sum = I.r + P.r + s.interaction_distance;
        if (d2 >= sum * sum) return;
        const auto key = std::make_tuple((ghost && P.id > I.id) ? 1 : 0, P.id, I.id);
        auto it = inter.find(key);
        if (it == inter.end()) {
            Inter n{};
            n.s = Springs{zero3(), zero3(), zero3()};
            if (std::get<0>(key) == 1) {
                // the ghost of the lower-id particle carries a copy of its
                // interaction with the real pair, history reversed
                // (BaseInteraction::copySwitchPointer, BaseInteraction.cc:340-356)
                auto pb = before.find(std::make_tuple(0, I.id, P.id));
                if (pb != before.end()) {
                    n.s.slide = -pb->second.second.slide;
                    n.s.roll = -pb->second.second.roll;
                    n.s.tors = -pb->second.second.tors;
                }
            }
            it = inter.emplace(key, n).first;
        }
        Inter& c = it->second;
        c.stamp = nt + 1;
        c.eval = evals;
        c.periodic = ghost;
        ContactGeom g;
        g.distance = std::sqrt(d2);
        g.n = branch / g.distance;
        g.overlap = P.r + I.r - g.distance;
        g.c = P.x - (P.r - 0.5 * g.overlap) * g.n;
        g.xp = P.x; g.vp = P.v; g.wp = P.w; g.inv_mass_p = P.invm; g.curv_p = 1.0 / P.r;
        g.xi = xi; g.vi = I.v; g.wi = I.w; g.inv_mass_i = I.invm; g.curv_i = 1.0 / I.r;
        g.i_is_wall = false;
        ContactOut out;
        evaluate_contact(s, g, c.s, cfg.time_step, out);
        c.overlap = g.overlap;
        c.force = out.force;
        c.energy = out.normal_stiffness_energy;
        P.F += out.force;
        P.T += out.torque - cross(P.x - g.c, out.force);
        if (!ghost) {
            I.F += -out.force;
            I.T += -out.torque + cross(I.x - g.c, out.force);
        }
    }

    bool wall_dist(int wi, V3 x, double radius, double& dist, V3& nrm) const
    {
        const dem_wall& w = walls[wi];
        const Q4 q{w.orientation[0], w.orientation[1], w.orientation[2], w.orientation[3]};
        const V3 wp = v3(w.position[0], w.position[1], w.position[2]);
        if (w.type == DEM_WALL_INFINITE) {
            dist = quat_plane_distance(q, x, wp);
            if (dist >= radius) return false;
            nrm = quat_axis(q);
            return true;
        }
        if (w.type == DEM_WALL_AXISYMMETRIC) { // AxisymmetricIntersectionOfWalls.cc:93-124
            const V3 po = x - wp;
            const V3 axis = quat_axis(q);
            const double a = dot(po, axis);
            V3 rad = po - axis * a;
            const double r = sqrt(len2(rad));
            V3 n2;
            if (!wgeo[wi].distance(v3(r, 0.0, a), radius, dist, n2)) return false;
            if (r != 0) rad = rad / r;
            nrm = axis * n2.z + rad * n2.x;
            return true;
        }
        // IntersectionOfWalls::getDistanceAndNormal(const BaseParticle&, ...) (:532-547)
        V3 nb;
        if (!wgeo[wi].distance(q_apply(q, x - wp, true), radius, dist, nb)) return false;
        nrm = q_apply(q, nb, false);
        return true;
    }

    void compute_forces()
    {
        ++evals;
        for (auto& q : p) { q.F = zero3(); q.T = zero3(); }
        const int n = (int)p.size();
        // removed particles (DeletionBoundary) take no part
        // candidate pairs: uniform grid over the box (exact FP64 predicate decides)
        double rmax = 0.0;
        for (auto& q : p) rmax = std::max(rmax, q.r);
        double dmax = 0.0;
        for (auto& s : species) dmax = std::max(dmax, s.interaction_distance);
        const double cs = 2.0 * rmax + dmax + 1e-12;
        double lo[3], hi[3];
        int dim[3];
        for (int k = 0; k < 3; ++k) {
            const bool per = (inst.periodic_mask >> k) & 1u;
            lo[k] = per ? inst.periodic_min[k] : inst.domain_min[k];
            hi[k] = per ? inst.periodic_max[k] : inst.domain_max[k];
            for (auto& q : p)
                if (!q.deleted) { lo[k] = std::min(lo[k], (&q.x.x)[k]); hi[k] = std::max(hi[k], (&q.x.x)[k]); }
            dim[k] = std::max(1, (int)std::floor((hi[k] - lo[k]) / cs));
        }
        auto cell_of = [&](V3 x, int k) {
            int c = (int)std::floor(((&x.x)[k] - lo[k]) / (hi[k] - lo[k]) * dim[k]);
            return std::max(0, std::min(dim[k] - 1, c));
        };
        std::vector<std::vector<int>> cells((size_t)dim[0] * dim[1] * dim[2]);
        for (int i = 0; i < n; ++i) {
            if (p[i].deleted) continue;
            const V3 x = p[i].x;
            cells[((size_t)cell_of(x, 2) * dim[1] + cell_of(x, 1)) * dim[0] + cell_of(x, 0)].push_back(i);
        }
        std::vector<int> cand;
        for (int i = 0; i < n; ++i) {
            if (p[i].deleted) continue;
            cand.clear();
            int c[3];
            for (int k = 0; k < 3; ++k) c[k] = cell_of(p[i].x, k);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        int cc[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
                        bool ok = true;
                        for (int k = 0; k < 3; ++k) {
                            if (cc[k] < 0 || cc[k] >= dim[k]) {
                                if ((inst.periodic_mask >> k) & 1u)
                                    cc[k] = (cc[k] + dim[k]) % dim[k];
                                else
                                    ok = false;
                            }
                        }
                        if (!ok) continue;
                        for (int j : cells[((size_t)cc[2] * dim[1] + cc[1]) * dim[0] + cc[0]]) cand.push_back(j);
                    }
            std::sort(cand.begin(), cand.end());
            cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
            for (int j : cand) {
                if (j == i) continue;
                Particle& A = p[i];
                Particle& B = p[j];
                if (A.fixed && B.fixed) continue;
                // image of B seen from A
                V3 xb = B.x;
                bool per = false;
                for (int k = 0; k < 3; ++k) {
                    if (!((inst.periodic_mask >> k) & 1u)) continue;
                    const double raw = (&A.x.x)[k] - (&xb.x)[k];
                    if (raw > half[k]) { (&xb.x)[k] = (&xb.x)[k] + L[k]; per = true; }
                    else if (raw < -half[k]) { (&xb.x)[k] = (&xb.x)[k] - L[k]; per = true; }
                }
                if (per) {
                    pair(A, B, xb, true); // A real, B's ghost
                } else if (A.id < B.id) {
                    pair(A, B, B.x, false);
                }
            }
        }
        // body forces
        for (auto& q : p) {
            if (q.fixed) continue;
            const double m = 1.0 / q.invm;
            q.F += v3(inst.gravity[0], inst.gravity[1], inst.gravity[2]) * m - cfg.background_drag * q.v;
        }
        // walls
        for (int w = 0; w < (int)walls.size(); ++w) {
            for (auto& q : p) {
                if (q.fixed) continue;
                const dem_wall& wall = walls[w];
                const dem_species_pair& s = sp(q.species, wall.species);
                double dist;
                V3 nrm;
                if (!wall_dist(w, q.x, q.r + s.interaction_distance, dist, nrm)) continue;
                const auto key = std::make_tuple(2, q.id, w);
                auto it = inter.find(key);
                if (it == inter.end()) {
                    Inter n{};
                    n.s = Springs{zero3(), zero3(), zero3()};
                    it = inter.emplace(key, n).first;
                }
                Inter& c = it->second;
                c.stamp = nt + 1;
        c.eval = evals;
                c.periodic = false;
                ContactGeom g;
                g.n = -nrm;
                g.distance = dist;
                g.overlap = q.r - dist;
                g.c = q.x - (q.r - 0.5 * g.overlap) * g.n;
                g.xp = q.x; g.vp = q.v; g.wp = q.w; g.inv_mass_p = q.invm; g.curv_p = 1.0 / q.r;
                g.xi = v3(wall.position[0], wall.position[1], wall.position[2]);
                g.vi = v3(wall.velocity[0], wall.velocity[1], wall.velocity[2]);
                g.wi = v3(wall.angular_velocity[0], wall.angular_velocity[1], wall.angular_velocity[2]);
                g.inv_mass_i = 0.0; g.curv_i = 0.0; g.i_is_wall = true;
                ContactOut out;
                evaluate_contact(s, g, c.s, cfg.time_step, out);
                c.overlap = g.overlap;
                c.force = out.force;
                c.energy = out.normal_stiffness_energy;
                q.F += out.force;
                q.T += out.torque - cross(q.x - g.c, out.force);
            }
        }
    }

    // Springs and stamps of the lower-id views of periodic pairs before an
    // evaluation (see periodic_handover).
    std::map<std::tuple<int, int, int>, std::pair<unsigned, Springs>> before;

    void snapshot_periodic()
    {
        before.clear();
        for (auto& kv : inter)
            if (std::get<0>(kv.first) == 0)
                before[kv.first] = {kv.second.stamp, kv.second.s};
    }

    // removeDuplicatePeriodicParticles: keep the lower-id particle's view of a
    // periodic pair; the other view restarts from the reversed spring. When the
    // real-real interaction carries the same stamp as the new view (the first
    // time step after initialiseSolve, whose stamps coincide), the reference
    // keeps the old interaction and drops this evaluation's spring update
    // (InteractionHandler.cc:339-352).
    void periodic_handover()
    {
        for (auto& kv : inter) {
            // the lower-id view of a pair that is periodic in this evaluation
            if (std::get<0>(kv.first) != 0 || !kv.second.periodic || kv.second.eval != evals) continue;
            const int a = std::get<1>(kv.first), b = std::get<2>(kv.first);
            auto pb = before.find(kv.first);
            if (pb != before.end() && pb->second.first == kv.second.stamp) kv.second.s = pb->second.second;
            auto other = inter.find(std::make_tuple(1, b, a));
            if (other == inter.end()) continue;
            other->second.s.slide = -kv.second.s.slide;
            other->second.s.roll = -kv.second.s.roll;
            other->second.s.tors = -kv.second.s.tors;
        }
    }

    // DeletionBoundary::checkBoundaryAfterParticleMoved (DeletionBoundary.cc:109-126):
    // the particle and its interactions leave the simulation
    std::vector<dem_deletion_boundary> dels;
    void delete_particles()
    {
        for (auto& q : p) {
            if (q.deleted) continue;
            bool gone = false;
            for (const auto& b : dels) {
                const double sf = 1. / std::sqrt(b.normal[0] * b.normal[0] + b.normal[1] * b.normal[1] +
                                                 b.normal[2] * b.normal[2]); // DeletionBoundary::set
                const double nx = b.normal[0] * sf, ny = b.normal[1] * sf, nz = b.normal[2] * sf;
                if (b.distance * sf - (q.x.x * nx + q.x.y * ny + q.x.z * nz) < 0) gone = true;
            }
            if (!gone) continue;
            q.deleted = true;
            q.fixed = true;
            q.invm = 0.0;
            q.v = zero3();
            q.w = zero3();
            for (auto it = inter.begin(); it != inter.end();) {
                const int kind = std::get<0>(it->first), a = std::get<1>(it->first), b = std::get<2>(it->first);
                if (a == q.id || (kind != 2 && b == q.id))
                    it = inter.erase(it);
                else
                    ++it;
            }
        }
    }

    // ---- insertion ---------------------------------------------------------
    std::vector<InsBoundary> ins;
    RefRng rng;                   // DPMBase::random
    std::vector<int> free_rows;   // input rows of radius 0, in row order
    size_t next_free = 0;
    double time = 0.0;            // DPMBase::time_
    double grid_rmax = 0.0;       // the largest radius the reference's HGrid was built for
    bool grid_fresh = false;      // a placement in this step rebuilt it
    bool no_row = false;

    double max_idist(int a) const
    {
        double m = 0.0;
        for (int b = 0; b < inst.n_species; ++b) m = std::max(m, sp(a, b).interaction_distance);
        return m;
    }

    // DPMBase::checkParticleForInteractionLocal for a candidate of radius r
    // and species a at x: no wall, then no particle, within reach
    bool free_at(V3 x, double r, int a) const
    {
        for (int w = 0; w < (int)walls.size(); ++w) {
            if (walls[w].type == DEM_WALL_TRIANGLE) continue;
            double dist;
            V3 nrm;
            if (wall_dist(w, x, r + sp(a, walls[w].species).interaction_distance, dist, nrm)) return false;
        }
        for (const auto& q : p) {
            if (q.deleted) continue;
            if (q.wrapped && !grid_fresh) continue; // filed in the HGrid on the far side
            const double X = x.x - q.x.x, Y = x.y - q.x.y, Z = x.z - q.x.z;
            const double sum = r + q.r + sp(a, q.species).interaction_distance;
            if (X * X + Y * Y + Z * Z < sum * sum) return false;
        }
        return true;
    }

    // DPMBase::checkParticleForInteractionLocalPeriodic: the candidate and its
    // copies, made per periodic boundary within the largest reach
    bool insertable(V3 x, double r, int a) const
    {
        std::vector<V3> copies;
        double largest = 0.0; // ParticleHandler::getLargestParticle()->getMaxInteractionRadius()
        bool any = false;
        for (const auto& q : p)
            if (!q.deleted) {
                largest = std::max(largest, q.r + max_idist(q.species) * 0.5);
                any = true;
            }
        for (int k = 0; k < 3 && any; ++k) {
            if (!((inst.periodic_mask >> k) & 1u)) continue;
            const double left = inst.periodic_min[k], right = inst.periodic_max[k];
            const double maxDistance = (r + max_idist(a) * 0.5) + largest;
            auto dist = [&](V3 y) { const double c = (&y.x)[k]; return std::min(c - left, right - c); };
            auto shift = [&](V3& y) {
                double& c = (&y.x)[k];
                c = (right - c > c - left) ? c + (right - left) : c - (right - left);
            };
            for (int i = (int)copies.size() - 1; i >= 0; --i)
                if (dist(copies[i]) < maxDistance) {
                    copies.push_back(copies[i]);
                    shift(copies.back());
                }
            if (dist(x) < maxDistance) {
                copies.push_back(x);
                shift(copies.back());
            }
        }
        if (!free_at(x, r, a)) return false;
        for (const V3& y : copies)
            if (!free_at(y, r, a)) return false;
        return true;
    }

    void insert()
    {
        const double next_time = time + cfg.time_step; // DPMBase::getNextTime
        grid_fresh = false;
        for (auto& B : ins) {
            const dem_insertion_boundary& b = B.b;
            auto generate = [&]() { // InsertionBoundary::generateParticle
                rng.draw(0, 1);
                B.p0_r = B.draw_radius();
                B.has_p0 = true;
            };
            unsigned failed = 0;
            while (failed <= (unsigned)b.max_failed && B.volume < b.volume_flow_rate * next_time + b.initial_volume) {
                if (!B.has_p0) generate();
                while (true) {
                    const double r = B.p0_r;
                    V3 x, v;
                    if (b.kind == DEM_INSERTION_CHUTE) {
                        x.x = b.pos_min[0] + r;
                        x.y = rng.draw(b.pos_min[1] - r, b.pos_max[1] + r);
                        x.z = rng.draw(b.pos_min[2] - r, b.pos_max[2] + r + b.fixed_particle_radius);
                        const double u = b.inflow_velocity, var = b.inflow_velocity_variance;
                        v.x = u * rng.draw(-var, var) + u;
                        v.y = u * rng.draw(-var, var);
                        v.z = u * rng.draw(-var, var);
                    } else {
                        x.x = rng.draw(b.pos_min[0], b.pos_max[0]);
                        x.y = rng.draw(b.pos_min[1], b.pos_max[1]);
                        x.z = rng.draw(b.pos_min[2], b.pos_max[2]);
                        v.x = rng.draw(b.vel_min[0], b.vel_max[0]);
                        v.y = rng.draw(b.vel_min[1], b.vel_max[1]);
                        v.z = rng.draw(b.vel_min[2], b.vel_max[2]);
                    }
                    if (insertable(x, r, b.species)) {
                        if (next_free >= free_rows.size()) {
                            no_row = true;
                            return;
                        }
                        Particle& q = p[free_rows[next_free++]];
                        q.x = x;
                        q.v = v;
                        q.w = zero3();
                        q.q = Q4{1.0, 0.0, 0.0, 0.0};
                        q.r = r;
                        // BaseParticle::computeMass (BaseParticle.cc:874-883), getVolume (:147-166)
                        const double pi = 3.1415926535897932384626433832795;
                        q.invm = 1.0 / (4.0 / 3.0 * pi * r * r * r * b.density);
                        q.invI = 1.0 / (.4 * (1.0 / q.invm) * (r * r));
                        q.species = b.species;
                        q.fixed = false;
                        q.deleted = false;
                        q.wrapped = false;
                        q.F = q.T = zero3();
                        failed = 0;
                        ++B.inserted;
                        B.volume += 4.0 / 3.0 * pi * r * r * r;
                        if (r > grid_rmax) { // HGrid::insertParticleToHgrid: too large, rebuild
                            grid_rmax = r;
                            grid_fresh = true;
                        }
                        generate();
                        break;
                    }
                    ++failed;
                    if (failed > (unsigned)b.max_failed) break;
                }
            }
        }
    }

    // Chute::addFlowParticlesCompactly with Chute::createFlowParticle
    // (Kernel/Chute.cc:1083-1115): candidates until the handler holds N
    // particles; a rejected one raises the inflow height. Returns false when
    // the free rows ran out.
    bool chute_fill(const dem_chute_fill& f, double& height)
    {
        unsigned n_objects = 0;
        for (const auto& q : p) n_objects += q.deleted ? 0u : 1u;
        const double r_in = 0.5 * (f.min_radius + f.max_radius); // getInflowParticleRadius
        const unsigned N = n_objects + f.x_max * f.y_max * height / (r_in * r_in * r_in) / 8;
        unsigned size = n_objects;
        while (size < N) {
            const double r = rng.draw(f.min_radius, f.max_radius);
            // the Vec3D constructor's arguments, evaluated last to first by g++
            const double z = rng.draw(f.z_min + r + f.fixed_particle_radius, height);
            const double y = rng.draw(f.y_min + r, f.y_max - r);
            const double x = rng.draw(f.x_min + r, f.x_max - r);
            if (insertable(v3(x, y, z), r, f.species)) {
                if (next_free >= free_rows.size()) return false;
                Particle& q = p[free_rows[next_free++]];
                q.x = v3(x, y, z);
                q.v = zero3();
                q.w = zero3();
                q.q = Q4{1.0, 0.0, 0.0, 0.0};
                q.r = r;
                const double pi = 3.1415926535897932384626433832795;
                q.invm = 1.0 / (4.0 / 3.0 * pi * r * r * r * f.density);
                q.invI = 1.0 / (.4 * (1.0 / q.invm) * (r * r));
                q.species = f.species;
                q.fixed = false;
                q.deleted = false;
                q.F = q.T = zero3();
                ++size;
            } else {
                height = height + .0001 * f.max_radius; // Chute::setInflowHeight
            }
        }
        return true;
    }

    void erase_old(unsigned current)
    {
        for (auto it = inter.begin(); it != inter.end();) {
            if (it->second.stamp <= current)
                it = inter.erase(it);
            else
                ++it;
        }
    }
};

} // namespace

static int g_report_handler = 0;
static std::vector<dem_deletion_boundary> g_deletions;
static std::vector<dem_insertion_boundary> g_insertions;
static unsigned long g_insertion_seed = 0;
static std::vector<long long> g_inserted;
static dem_chute_fill g_fill;
static bool g_fill_set = false;
static double g_fill_height = 0.0;
static std::vector<double> g_inserted_volume;

extern "C" {

// 0: report the contacts of the last force evaluation (what the engine
// records); 1: report every interaction the reference's handler still holds
// after the step (after step 0 this includes interactions of the initial
// evaluation that step 0 did not touch: both carry time stamp 1).
void oracle_set_contact_report(int mode) { g_report_handler = mode; }

// DeletionBoundary planes of the next oracle_run (the instance field is ignored).
void oracle_set_deletion(const dem_deletion_boundary* b, int n) { g_deletions.assign(b, b + n); }

// Insertion boundaries of the next oracle_run (instance fields ignored) and
// the seed of DPMBase::random; input rows of radius 0 are then free rows.
void oracle_set_insertion(const dem_insertion_boundary* b, int n, unsigned long long seed)
{
    g_insertions.assign(b, b + n);
    g_insertion_seed = (unsigned long)seed;
}

// Chute::addFlowParticlesCompactly before the next oracle_run's initial force
// evaluation (set = 0: none), from DPMBase::random seeded with `seed`; input
// rows of radius 0 are the free rows. oracle_chute_fill_height: the inflow
// height it ended with.
void oracle_set_chute_fill(const dem_chute_fill* f, int set, unsigned long long seed)
{
    if (f) g_fill = *f;
    g_fill_set = set != 0;
    g_insertion_seed = (unsigned long)seed;
}
double oracle_chute_fill_height() { return g_fill_height; }

// Particles and volume each insertion boundary placed in the last oracle_run;
// returns the number of boundaries, -1 if a placement found no free row.
int oracle_insertion_counts(long long* inserted, double* volume, int capacity)
{
    const int n = (int)g_inserted.size();
    for (int k = 0; k < n && k < capacity; ++k) {
        inserted[k] = g_inserted[k];
        volume[k] = g_inserted_volume[k];
    }
    return n;
}

// Runs nsteps reference time steps from the given state (after the initial
// force evaluation of DPMBase::initialiseSolve) and returns the final state
// (caller order), the forces of the last evaluation and the live contacts.
int oracle_run(const dem_config* cfg, const dem_instance_desc* inst, const dem_species_pair* species, int nspecies,
               const dem_wall* walls, int nwalls, const dem_particles_soa* in, const dem_contacts_soa* contacts_in,
               int nsteps, dem_particles_soa* out, double* force, double* torque, dem_contacts_soa* contacts_out,
               int64_t contacts_capacity, int64_t* contacts_count)
{
    for (int w = 0; w < nwalls; ++w) // triangle walls are checked against the reference build itself
        if (walls[w].type == DEM_WALL_TRIANGLE) return -2;
    Sim S;
    S.cfg = *cfg;
    S.inst = *inst;
    S.species.assign(species, species + nspecies);
    S.walls.assign(walls, walls + nwalls);
    S.dels = g_deletions;
    S.wgeo.resize(nwalls);
    for (int w = 0; w < nwalls; ++w)
        if (walls[w].type != DEM_WALL_INFINITE) S.wgeo[w].build(walls[w]);
    for (int k = 0; k < 3; ++k) {
        S.L[k] = inst->periodic_max[k] - inst->periodic_min[k];
        S.half[k] = 0.5 * S.L[k];
    }
    const int64_t n = in->n;
    S.p.resize(n);
    for (int64_t i = 0; i < n; ++i) {
        Particle& q = S.p[i];
        q.x = v3(in->position[3 * i], in->position[3 * i + 1], in->position[3 * i + 2]);
        q.v = v3(in->velocity[3 * i], in->velocity[3 * i + 1], in->velocity[3 * i + 2]);
        q.w = in->angular_velocity ? v3(in->angular_velocity[3 * i], in->angular_velocity[3 * i + 1],
                                        in->angular_velocity[3 * i + 2])
                                   : zero3();
        q.q = in->orientation ? Q4{in->orientation[4 * i], in->orientation[4 * i + 1], in->orientation[4 * i + 2],
                                   in->orientation[4 * i + 3]}
                              : Q4{1.0, 0.0, 0.0, 0.0};
        q.r = in->radius[i];
        q.invm = in->inv_mass[i];
        q.invI = in->inv_inertia ? in->inv_inertia[i] : 0.0;
        q.species = in->species[i];
        q.id = in->id[i];
        q.fixed = q.invm == 0.0;
        q.F = q.T = zero3();
        if ((!g_insertions.empty() || g_fill_set) && q.r == 0.0) { // a free row: no particle until one is placed
            q.deleted = true;
            q.fixed = true;
            q.invm = 0.0;
            S.free_rows.push_back((int)i);
        } else {
            S.grid_rmax = std::max(S.grid_rmax, q.r);
        }
    }
    S.rng = RefRng(g_insertion_seed);
    for (const auto& b : g_insertions) {
        InsBoundary B;
        B.b = b;
        B.psd_rng = RefRng((unsigned long)b.psd_seed);
        S.ins.push_back(B);
    }
    std::map<int, int> index_of;
    for (int64_t i = 0; i < n; ++i) index_of[S.p[i].id] = (int)i;
    if (contacts_in) {
        for (int64_t r = 0; r < contacts_in->n; ++r) {
            Inter c{};
            const double* s = contacts_in->springs + 9 * r;
            c.s = Springs{v3(s[0], s[1], s[2]), v3(s[3], s[4], s[5]), v3(s[6], s[7], s[8])};
            c.stamp = 0;
            const bool wall = contacts_in->is_wall && contacts_in->is_wall[r];
            const bool per = contacts_in->periodic && contacts_in->periodic[r];
            if (wall) {
                S.inter[std::make_tuple(2, contacts_in->id_p[r], contacts_in->id_i[r])] = c;
            } else if (per) {
                c.periodic = true;
                S.inter[std::make_tuple(0, contacts_in->id_p[r], contacts_in->id_i[r])] = c;
                Inter o = c;
                o.s.slide = -c.s.slide; o.s.roll = -c.s.roll; o.s.tors = -c.s.tors;
                S.inter[std::make_tuple(1, contacts_in->id_i[r], contacts_in->id_p[r])] = o;
            } else {
                S.inter[std::make_tuple(0, contacts_in->id_p[r], contacts_in->id_i[r])] = c;
            }
        }
    }
    if (g_fill_set) { // Chute::setupInitialConditions runs before the first force evaluation
        double height = g_fill.inflow_height;
        if (!S.chute_fill(g_fill, height)) return -3;
        g_fill_height = height;
    }
    // DPMBase::initialiseSolve: numberOfTimeSteps_ = 0, one force evaluation
    S.nt = 0;
    S.snapshot_periodic();
    S.compute_forces();
    S.periodic_handover();
    for (int step = 0; step < nsteps; ++step) {
        S.integrate_before();
        S.wrap();
        S.delete_particles();
        if (!S.ins.empty()) {
            S.insert();
            if (S.no_row) return -3;
        }
        S.time += S.cfg.time_step; // the time the reference reaches at the end of the step
        S.snapshot_periodic();
        S.compute_forces();
        S.periodic_handover();
        S.integrate_after();
        S.erase_old(S.nt);
        S.nt += 1;
    }
    g_inserted.clear();
    g_inserted_volume.clear();
    for (const auto& B : S.ins) {
        g_inserted.push_back(B.inserted);
        g_inserted_volume.push_back(B.volume);
    }
    if (out) {
        for (int64_t i = 0; i < n; ++i) {
            const Particle& q = S.p[i];
            if (out->position) { out->position[3 * i] = q.x.x; out->position[3 * i + 1] = q.x.y; out->position[3 * i + 2] = q.x.z; }
            if (out->velocity) { out->velocity[3 * i] = q.v.x; out->velocity[3 * i + 1] = q.v.y; out->velocity[3 * i + 2] = q.v.z; }
            if (out->angular_velocity) {
                out->angular_velocity[3 * i] = q.w.x; out->angular_velocity[3 * i + 1] = q.w.y; out->angular_velocity[3 * i + 2] = q.w.z;
            }
            if (out->orientation) {
                out->orientation[4 * i] = q.q.q0; out->orientation[4 * i + 1] = q.q.q1;
                out->orientation[4 * i + 2] = q.q.q2; out->orientation[4 * i + 3] = q.q.q3;
            }
            if (out->instance) out->instance[i] = q.deleted ? -1 : 0;
            if (out->radius) out->radius[i] = q.r;
            if (out->inv_mass) out->inv_mass[i] = q.invm;
            if (out->inv_inertia) out->inv_inertia[i] = q.invI;
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        const Particle& q = S.p[i];
        if (force) { force[3 * i] = q.F.x; force[3 * i + 1] = q.F.y; force[3 * i + 2] = q.F.z; }
        if (torque) { torque[3 * i] = q.T.x; torque[3 * i + 1] = q.T.y; torque[3 * i + 2] = q.T.z; }
    }
    // live contacts as the reference keeps them after the step
    int64_t cnt = 0;
    for (const auto& kv : S.inter) {
        const int kind = std::get<0>(kv.first), a = std::get<1>(kv.first), b = std::get<2>(kv.first);
        if (g_report_handler) {
            // every interaction the reference's InteractionHandler still holds
            const unsigned last_stamp = nsteps > 0 ? (unsigned)nsteps : 1u;
            if (kv.second.stamp != last_stamp) continue;
        } else if (kv.second.eval != S.evals) {
            continue; // only contacts of the last force evaluation
        }
        if (kind == 1) continue; // the higher-id view of a periodic pair is not kept
        if (contacts_out && cnt < contacts_capacity) {
            contacts_out->id_p[cnt] = a;
            contacts_out->id_i[cnt] = b;
            if (contacts_out->is_wall) contacts_out->is_wall[cnt] = kind == 2;
            if (contacts_out->periodic) contacts_out->periodic[cnt] = kind == 0 && kv.second.periodic;
            if (contacts_out->overlap) contacts_out->overlap[cnt] = kv.second.overlap;
            if (contacts_out->force) {
                contacts_out->force[3 * cnt] = kv.second.force.x;
                contacts_out->force[3 * cnt + 1] = kv.second.force.y;
                contacts_out->force[3 * cnt + 2] = kv.second.force.z;
            }
            if (contacts_out->springs) {
                const Springs& s = kv.second.s;
                const double v[9] = {s.slide.x, s.slide.y, s.slide.z, s.roll.x, s.roll.y, s.roll.z,
                                     s.tors.x, s.tors.y, s.tors.z};
                std::memcpy(contacts_out->springs + 9 * cnt, v, sizeof(v));
            }
        }
        ++cnt;
    }
    if (contacts_count) *contacts_count = cnt;
    if (contacts_out) contacts_out->n = std::min(cnt, contacts_capacity);
    return 0;
}

} // extern "C"
