// dem_walls.cuh -- wall geometry on the device.
//
// InfiniteWall::getDistanceAndNormal (Kernel/Walls/InfiniteWall.cc:151-175):
// distance from Quaternion::getDistance of the wall's orientation and
// position, normal = Quaternion::getAxis.
// AxisymmetricIntersectionOfWalls::getDistanceAndNormal
// (Kernel/Walls/AxisymmetricIntersectionOfWalls.cc:93-124) maps the particle
// to the wall's axis frame (r, 0, axial) and evaluates
// IntersectionOfWalls::getDistanceAndNormal (IntersectionOfWalls.cc:567-700)
// on the half-planes stored in faces[].
#pragma once
#include "dem_math.cuh"
#include "../../include/dem_b200.h"

namespace dem {

__device__ __forceinline__ Q4 wall_q(const dem_wall& w)
{
    return Q4{w.orientation[0], w.orientation[1], w.orientation[2], w.orientation[3]};
}

// Quaternion::rotateBack (Quaternion.cc): lab -> body frame, R^T p.
__device__ __forceinline__ V3 quat_rotate_back(Q4 q, V3 p)
{
    const double q00 = q.q0 * q.q0, q11 = q.q1 * q.q1, q22 = q.q2 * q.q2, q33 = q.q3 * q.q3;
    const double q01 = q.q0 * q.q1, q02 = q.q0 * q.q2, q03 = q.q0 * q.q3;
    const double q12 = q.q1 * q.q2, q13 = q.q1 * q.q3, q23 = q.q2 * q.q3;
    return V3{(q00 + q11 - q22 - q33) * p.x + 2.0 * (q12 + q03) * p.y + 2.0 * (q13 - q02) * p.z,
              2.0 * (q12 - q03) * p.x + (q00 - q11 + q22 - q33) * p.y + 2.0 * (q23 + q01) * p.z,
              2.0 * (q13 + q02) * p.x + 2.0 * (q23 - q01) * p.y + (q00 - q11 - q22 + q33) * p.z};
}

// Quaternion::rotate (Quaternion.cc): body -> lab frame, R p.
__device__ __forceinline__ V3 quat_rotate_vec(Q4 q, V3 p)
{
    const double q00 = q.q0 * q.q0, q11 = q.q1 * q.q1, q22 = q.q2 * q.q2, q33 = q.q3 * q.q3;
    const double q01 = q.q0 * q.q1, q02 = q.q0 * q.q2, q03 = q.q0 * q.q3;
    const double q12 = q.q1 * q.q2, q13 = q.q1 * q.q3, q23 = q.q2 * q.q3;
    return V3{(q00 + q11 - q22 - q33) * p.x + 2.0 * (q12 - q03) * p.y + 2.0 * (q13 + q02) * p.z,
              2.0 * (q12 + q03) * p.x + (q00 - q11 + q22 - q33) * p.y + 2.0 * (q23 - q01) * p.z,
              2.0 * (q13 - q02) * p.x + 2.0 * (q23 + q01) * p.y + (q00 - q11 - q22 + q33) * p.z};
}

// Intersection of half-planes in the (r, 0, a) plane; a point is inside when
// it is on the negative side of every face normal. Returns the distance to
// the closest face (with edge/corner handling as in IntersectionOfWalls).
__device__ __forceinline__ bool intersection_distance(const dem_wall& w, V3 p, double wall_radius, double& distance, V3& normal);

__device__ __forceinline__ bool wall_distance(const dem_wall& w, V3 x, double wall_radius, double& dist, V3& normal)
{
    if (w.type == DEM_WALL_INFINITE) {
        const Q4 q = wall_q(w);
        dist = quat_plane_distance(q, x, v3(w.position[0], w.position[1], w.position[2]));
        if (dist >= wall_radius) return false;
        normal = quat_axis(q);
        return true;
    }
    if (w.type == DEM_WALL_AXISYMMETRIC) {
        // AxisymmetricIntersectionOfWalls::getDistanceAndNormal
        const Q4 q = wall_q(w);
        V3 pos = x - v3(w.position[0], w.position[1], w.position[2]);
        pos = quat_rotate_back(q, pos);
        // the wall axis is the body-frame x axis after rotateBack (orientation of (1,0,0))
        const V3 axis = v3(1.0, 0.0, 0.0);
        const double a = dot(pos, axis);
        const V3 radial = pos - a * axis;
        const double rr = len(radial);
        const V3 rp = v3(rr, 0.0, a);
        double d;
        V3 nrz;
        if (!intersection_distance(w, rp, wall_radius, d, nrz)) return false;
        dist = d;
        // map the (r, 0, a) normal back: radial component along the radial unit vector
        V3 nb;
        if (rr != 0.0) {
            const V3 ur = radial / rr;
            nb = nrz.x * ur + nrz.z * axis;
        } else {
            nb = nrz.z * axis;
        }
        normal = quat_rotate_vec(q, nb);
        return true;
    }
    return false;
}

__device__ __forceinline__ bool intersection_distance(const dem_wall& w, V3 p, double wall_radius, double& distance, V3& normal)
{
    // Signed distance to each face: faces[k] = (nx, ny, nz, px, py, pz), outward normal n,
    // the wall occupies {x : dot(x - p, n) <= 0 for all faces} complement... The
    // particle is in contact with the face whose distance is largest (least negative
    // penetration) among faces that bound the wall.
    const int nf = w.n_faces;
    double dmax = -1e300;
    int imax = -1;
    for (int k = 0; k < nf; ++k) {
        const V3 n = v3(w.faces[k][0], w.faces[k][1], w.faces[k][2]);
        const V3 q = v3(w.faces[k][3], w.faces[k][4], w.faces[k][5]);
        const double dk = dot(q - p, n);
        if (dk > dmax) {
            dmax = dk;
            imax = k;
        }
    }
    if (imax < 0 || dmax >= wall_radius) return false;
    distance = dmax;
    normal = v3(w.faces[imax][0], w.faces[imax][1], w.faces[imax][2]);
    return true;
}

} // namespace dem
