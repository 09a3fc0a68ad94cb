// dem_laws.cuh -- contact force laws evaluated per contact on the device.
//
// One function evaluates normal law + friction law for one contact, in the
// order Interaction<N,F,A>::computeForce uses (Kernel/Interactions/Interaction.h:312-317):
//   normal:   LinearViscoelasticInteraction::computeNormalForce   (LinearViscoelasticInteraction.cc:105-135)
//             HertzianViscoelasticInteraction::computeNormalForce (HertzianViscoelasticInteraction.cc:106-141)
//   friction: SlidingFrictionInteraction::computeFrictionForce    (SlidingFrictionInteraction.cc:106-193)
//             FrictionInteraction::computeFrictionForce           (FrictionInteraction.cc:108-232)
//             MindlinInteraction::computeFrictionForce            (MindlinInteraction.cc:279-344)
//             MindlinRollingTorsionInteraction::computeFrictionForce (MindlinRollingTorsionInteraction.cc:109-208)
// The spring history (sliding, rolling, torsion) is read and written through
// the Springs struct; the caller owns where it lives in memory.
#pragma once
#include "dem_math.cuh"
#include "../../include/dem_b200.h"

namespace dem {

struct Springs {
    V3 slide, roll, tors;
};

// Geometry and kinematics of one contact. P is the body the force acts on
// (lower-id particle, or the particle of a particle-wall contact); I is the
// other body. For a wall, inv_mass_i == 0 and curvature_i == 0.
struct ContactGeom {
    V3 n;            // unit normal, from I towards P
    double overlap;  // r_P + r_I - distance (particle-particle) or r - distance (wall)
    double distance;
    V3 c;            // contact point
    V3 xp, vp, wp;   // P: position, velocity, angular velocity
    V3 xi, vi, wi;   // I
    double curv_p, curv_i;       // 1/r, 0 for a wall (BaseParticle.h:300-301, BaseInteractable.h:414)
    double inv_mass_p, inv_mass_i;
    bool i_is_wall;
};

struct ContactOut {
    V3 force;            // force on P
    V3 torque;           // interaction torque (rolling/torsion), on P
    V3 tangential;       // the friction force (getTangentialForce), part of force
    double abs_normal_force;
    double normal_stiffness_energy; // elastic energy of this contact (for balances)
};

// Relative velocity at the contact point: v_P(c) - v_I(c) with
// v(c) = v - (c - x) x omega (BaseInteractable::getVelocityAtContact, BaseInteractable.cc:375-378).
__device__ __host__ __forceinline__ V3 velocity_at_contact(V3 v, V3 x, V3 w, V3 c)
{
    return v - cross(c - x, w);
}

__device__ __host__ __forceinline__ double sq(double a) { return a * a; }

// NLAW / FLAW fix the normal and friction law at compile time (-1: read them
// from the species pair at run time); the kernels instantiate the law pair a
// simulation uses so that unused branches cost neither registers nor code.
template <int NLAW = -1, int FLAW = -1>
__device__ __host__ __forceinline__ void evaluate_contact(const dem_species_pair& sp, const ContactGeom& g,
                                                          Springs& s, double dt, ContactOut& out)
{
    const int nl = NLAW >= 0 ? NLAW : sp.normal_law;
    const V3 vrel = velocity_at_contact(g.vp, g.xp, g.wp, g.c) - velocity_at_contact(g.vi, g.xi, g.wi, g.c);
    const double vn = dot(vrel, g.n);
    const double meff = 1.0 / (g.inv_mass_p + g.inv_mass_i);   // BaseInteraction.cc:810-816
    const double reff = 1.0 / (g.curv_p + g.curv_i);           // BaseInteraction.cc:793-799
    double abs_fn = 0.0;
    V3 force = zero3();
    V3 torque = zero3();
    V3 tangential = zero3();
    double kt0 = 0.0; // Mindlin tangential stiffness of this step
    out.normal_stiffness_energy = 0.0;

    // ---- normal force ----
    if (g.overlap > 0) {
        double fn;
        if (nl == DEM_NORMAL_HERTZIAN_VISCOELASTIC) {
            const double k = 4. / 3. * sp.elastic_modulus * sqrt(reff * g.overlap);
            const double diss = sp.dissipation * sqrt(meff * k);
            fn = k * g.overlap - diss * vn;
            // HertzianViscoelasticInteraction::getElasticEnergy: 2/5 k delta^2
            out.normal_stiffness_energy = 0.4 * k * g.overlap * g.overlap;
        } else {
            fn = sp.stiffness * g.overlap - sp.dissipation * vn;
            if (sp.constant_restitution) fn *= 2.0 * meff;
            out.normal_stiffness_energy = sp.constant_restitution ? meff * sp.stiffness * g.overlap * g.overlap
                                                                  : 0.5 * sp.stiffness * g.overlap * g.overlap;
        }
        abs_fn = fabs(fn);
        force = g.n * fn;
    }

    // ---- friction ----
    const int fl = FLAW >= 0 ? FLAW : sp.friction_law;
    if (abs_fn != 0.0 && fl != DEM_FRICTION_NONE) {
        if (fl == DEM_FRICTION_SLIDING || fl == DEM_FRICTION_ROLLING_TORSION) {
            // SlidingFrictionInteraction::computeFrictionForce
            if (sp.sliding_mu != 0.0) {
                const V3 vt = vrel - g.n * vn;
                if (sp.sliding_stiffness != 0.0) {
                    V3 sv;
                    if (g.i_is_wall) {
                        sv = vt;
                    } else {
                        sv = vt - (dot(s.slide, g.vp - g.vi) * g.n) / g.distance;
                    }
                    s.slide += sv * dt;
                    V3 ft = (-sp.sliding_stiffness) * s.slide - sp.sliding_dissipation * vt;
                    if (sp.constant_restitution) ft *= 2.0 * meff;
                    const double ft2 = len2(ft);
                    if (ft2 <= sq(sp.sliding_mu_static * abs_fn)) {
                        force += ft;
                    } else {
                        ft *= sp.sliding_mu * abs_fn / sqrt(ft2);
                        force += ft;
                        s.slide = -(ft + sp.sliding_dissipation * vt) / sp.sliding_stiffness;
                    }
                    tangential = ft;
                } else {
                    const double vt2 = len2(vt);
                    V3 ft;
                    if (vt2 * sq(sp.sliding_dissipation) <= sq(sp.sliding_mu_static * abs_fn))
                        ft = -sp.sliding_dissipation * vt;
                    else
                        ft = -(sp.sliding_mu * abs_fn / sqrt(vt2)) * vt;
                    force += ft;
                    tangential = ft;
                }
            }
            if (fl == DEM_FRICTION_ROLLING_TORSION) {
                // FrictionInteraction::computeFrictionForce (rolling and torsion part)
                if (sp.rolling_mu != 0.0 && sp.rolling_stiffness != 0.0) {
                    const double deff = 2.0 * reff;
                    const V3 vr = -deff * cross(g.n, g.wp - g.wi);
                    V3 rsv;
                    if (g.i_is_wall) {
                        rsv = vr;
                    } else {
                        const V3 rv = g.vp - g.vi;
                        rsv = vr - dot(s.roll, rv) / g.distance * g.n;
                    }
                    s.roll += rsv * dt;
                    V3 fr = -sp.rolling_stiffness * s.roll - sp.rolling_dissipation * vr;
                    if (sp.constant_restitution) fr *= 2.0 * meff;
                    const double fr2 = len2(fr);
                    if (!(fr2 <= sq(sp.rolling_mu_static * abs_fn))) {
                        fr *= sp.rolling_mu * abs_fn / sqrt(fr2);
                        s.roll = -(fr + sp.rolling_dissipation * vr) / sp.rolling_stiffness;
                    }
                    torque += deff * cross(g.n, fr);
                }
                if (sp.torsion_mu != 0.0 && sp.torsion_stiffness != 0.0) {
                    const double deff = 2.0 * reff;
                    const V3 vo = deff * dot(g.n, g.wp - g.wi) * g.n;
                    s.tors = dot(s.tors + vo * dt, g.n) * g.n;
                    V3 fo = -sp.torsion_stiffness * s.tors - sp.torsion_dissipation * vo;
                    if (sp.constant_restitution) fo *= 2.0 * meff;
                    const double fo2 = len2(fo);
                    if (!(fo2 <= sq(sp.torsion_mu_static * abs_fn))) {
                        fo *= sp.torsion_mu * abs_fn / sqrt(fo2);
                        s.tors = -(fo + sp.torsion_dissipation * vo) / sp.torsion_stiffness;
                    }
                    torque += deff * fo;
                }
            }
        } else {
            // MindlinInteraction::computeFrictionForce
            if (sp.sliding_mu != 0.0) {
                const V3 vt = vrel - g.n * vn;
                const double L = len(s.slide);
                if (L > 1e-10) {
                    s.slide -= dot(s.slide, g.n) * g.n;
                    s.slide *= L / len(s.slide);
                }
                s.slide += vt * dt;
                const double r1 = 1.0 * reff;
                kt0 = 8 * sp.shear_modulus * sqrt(r1 * g.overlap);
                const double sdc = sp.sliding_dissipation * sqrt(meff * kt0);
                V3 ft = -2.0 / 3.0 * kt0 * s.slide;
                if (len(ft) < sp.sliding_mu * abs_fn) {
                    ft -= sdc * vt;
                    force += ft;
                } else {
                    ft *= sp.sliding_mu * abs_fn / len(ft);
                    force += ft;
                    s.slide = -(ft / (2.0 / 3.0 * kt0));
                }
                tangential = ft;
            }
            if (fl == DEM_FRICTION_MINDLIN_ROLLING_TORSION) {
                if (sp.rolling_mu != 0.0) {
                    const double kr = kt0;
                    const double er = reff;
                    const V3 vr = -er * cross(g.n, g.wp - g.wi);
                    const double L = len(s.roll);
                    if (L > 1e-10) {
                        s.roll -= dot(s.roll, g.n) * g.n;
                        s.roll *= L / len(s.roll);
                    }
                    s.roll += vr * dt;
                    V3 fr = -kr * s.roll - sp.rolling_dissipation * vr;
                    const double fr2 = len2(fr);
                    if (!(fr2 <= sq(sp.rolling_mu_static * abs_fn))) {
                        fr *= sp.rolling_mu * abs_fn / sqrt(fr2);
                        s.roll = -(fr + sp.rolling_dissipation * vr) / kr;
                    }
                    torque += er * cross(g.n, fr);
                }
                if (sp.torsion_mu != 0.0) {
                    const double ko = kt0;
                    const double deff = 2.0 * reff;
                    const V3 vo = deff * dot(g.n, g.wp - g.wi) * g.n;
                    s.tors += dot(s.tors + vo * dt, g.n) * g.n;
                    V3 fo = -ko * s.tors - sp.torsion_dissipation * vo;
                    const double fo2 = len2(fo);
                    if (!(fo2 <= sq(sp.torsion_mu_static * abs_fn))) {
                        fo *= sp.torsion_mu * abs_fn / sqrt(fo2);
                        s.tors = -(fo + sp.torsion_dissipation * vo) / ko;
                    }
                    torque += deff * fo;
                }
            }
        }
    }
    out.force = force;
    out.torque = torque;
    out.tangential = tangential;
    out.abs_normal_force = abs_fn;
}

} // namespace dem
