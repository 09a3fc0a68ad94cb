// dem_walls.cuh -- wall geometry on the device (and its host-side set-up).
//
// InfiniteWall::getDistanceAndNormal (Kernel/Walls/InfiniteWall.cc:151-175):
// distance from Quaternion::getDistance of the wall's orientation and
// position, normal = Quaternion::getAxis.
//
// IntersectionOfWalls (Kernel/Walls/IntersectionOfWalls.cc): a set of
// half-spaces ("faces", each an InfiniteWall built by addObject(normal,
// point), :138-149); a particle touches the wall where it lies inside every
// face but within the interaction radius of the boundary. Faces, edge lines
// (A_, AB_) and corner points (C_) are precomputed on the host exactly as
// setPointsAndLines (:351-450) does, and the device evaluates the face /
// edge / corner selection of getDistanceAndNormal(Vec3D, ...) (:567-712).
// The plain IntersectionOfWalls maps the particle into the wall frame with
// Quaternion::rotateBack and the normal back with Quaternion::rotate
// (:532-547); AxisymmetricIntersectionOfWalls maps it to (r, 0, a) about the
// wall's axis (AxisymmetricIntersectionOfWalls.cc:93-124).
#pragma once
#include <cstring>

#include "dem_math.cuh"
#include "../../include/dem_b200.h"

namespace dem {

constexpr int WALL_PAIRS = DEM_MAX_WALL_FACES * (DEM_MAX_WALL_FACES - 1) / 2;
constexpr int WALL_TRIPLES = DEM_MAX_WALL_FACES * (DEM_MAX_WALL_FACES - 1) * (DEM_MAX_WALL_FACES - 2) / 6;

// Derived geometry of one intersection wall (unused for infinite walls).
struct WallGeom {
    double fq[DEM_MAX_WALL_FACES][4]; // face orientation (InfiniteWall::setNormal)
    double fp[DEM_MAX_WALL_FACES][3]; // face position
    double fn[DEM_MAX_WALL_FACES][3]; // face normal = Quaternion::getAxis(fq)
    double A[WALL_PAIRS][3];          // a point on the edge of faces (m, n)
    double AB[WALL_PAIRS][3];         // unit direction of that edge
    double C[WALL_TRIPLES][3];        // the corner of faces (l, m, n)
    // triangle walls
    double tvl[3][3];                 // vertices relative to the position (vertexInLabFrame_)
    double tv[3][3];                  // vertices in the lab frame (vertex_)
    double te[3][3];                  // unit edges v1-v0, v2-v1, v0-v2 (edge_)
    double ten[3][3];                 // unit in-plane edge normals (edgeNormal_)
    double tel[3];                    // edge lengths (edgeLength_)
    double tfn[3];                    // unit face normal (faceNormal_)
    double tlo[3], thi[3];            // bounding box of the vertices (vertexMin_, vertexMax_)
};

__host__ __device__ __forceinline__ Q4 wall_q(const dem_wall& w)
{
    return Q4{w.orientation[0], w.orientation[1], w.orientation[2], w.orientation[3]};
}

__host__ __device__ __forceinline__ V3 row3(const double* a) { return V3{a[0], a[1], a[2]}; }

// Rotation matrix entries of a unit quaternion with the reference's rounding
// (Quaternion::rotate / rotateBack, Quaternion.cc:570-640).
struct QRot {
    double q00, q01, q02, q03, q11, q12, q13, q22, q23, q33;
};

__host__ __device__ __forceinline__ QRot qrot(Q4 q)
{
    QRot r;
    r.q00 = q.q0 * q.q0;
    r.q01 = 2 * q.q0 * q.q1;
    r.q02 = 2 * q.q0 * q.q2;
    r.q03 = 2 * q.q0 * q.q3;
    r.q11 = q.q1 * q.q1;
    r.q12 = 2 * q.q1 * q.q2;
    r.q13 = 2 * q.q1 * q.q3;
    r.q22 = q.q2 * q.q2;
    r.q23 = 2 * q.q2 * q.q3;
    r.q33 = q.q3 * q.q3;
    return r;
}

// body -> lab (Quaternion::rotate)
__host__ __device__ __forceinline__ V3 quat_to_lab(Q4 q, V3 p)
{
    const QRot r = qrot(q);
    const double m00 = r.q00 + r.q11 - r.q22 - r.q33, m01 = r.q12 - r.q03, m02 = r.q13 + r.q02;
    const double m10 = r.q12 + r.q03, m11 = r.q00 - r.q11 + r.q22 - r.q33, m12 = r.q23 - r.q01;
    const double m20 = r.q13 - r.q02, m21 = r.q23 + r.q01, m22 = r.q00 - r.q11 - r.q22 + r.q33;
    return V3{m00 * p.x + m01 * p.y + m02 * p.z, m10 * p.x + m11 * p.y + m12 * p.z, m20 * p.x + m21 * p.y + m22 * p.z};
}

// lab -> body (Quaternion::rotateBack)
__host__ __device__ __forceinline__ V3 quat_to_body(Q4 q, V3 p)
{
    const QRot r = qrot(q);
    const double m00 = r.q00 + r.q11 - r.q22 - r.q33, m01 = r.q12 + r.q03, m02 = r.q13 - r.q02;
    const double m10 = r.q12 - r.q03, m11 = r.q00 - r.q11 + r.q22 - r.q33, m12 = r.q23 + r.q01;
    const double m20 = r.q13 + r.q02, m21 = r.q23 - r.q01, m22 = r.q00 - r.q11 - r.q22 + r.q33;
    return V3{m00 * p.x + m01 * p.y + m02 * p.z, m10 * p.x + m11 * p.y + m12 * p.z, m20 * p.x + m21 * p.y + m22 * p.z};
}

__host__ __device__ __forceinline__ double face_distance(const WallGeom& g, unsigned k, V3 x)
{
    return quat_plane_distance(Q4{g.fq[k][0], g.fq[k][1], g.fq[k][2], g.fq[k][3]}, x, row3(g.fp[k]));
}

// IntersectionOfWalls::getDistanceAndNormal(const Vec3D&, ...): the face with
// the largest signed distance decides, unless the closest point on it lies
// outside a second (edge: distance to the line A + t AB) or a third face
// (corner: distance to C). Face, edge and corner indices and the NaN
// fall-through (the corner of three faces whose normals are coplanar has no
// finite C) follow the reference.
__host__ __device__ __forceinline__ bool intersection_distance(const WallGeom& g, int nf, V3 position, double R,
                                                               double& distance, V3& normal)
{
    if (nf <= 0) return false;
    distance = -1e20;
    double distance2 = -1e20, distance3 = -1e20;
    unsigned id = 0, id2 = 0, id3 = 0;
    for (unsigned i = 0; i < (unsigned)nf; ++i) {
        const double dc = face_distance(g, i, position);
        if (dc >= R) return false;
        if (dc > distance) {
            if (distance > -R) {
                if (distance2 > -R) {
                    distance3 = distance2;
                    id3 = id2;
                }
                distance2 = distance;
                id2 = id;
            }
            distance = dc;
            id = i;
        } else if (dc < -R) {
            continue;
        } else if (dc > distance2) {
            if (distance2 > -R) {
                distance3 = distance2;
                id3 = id2;
            }
            distance2 = dc;
            id2 = i;
        } else if (dc > distance3) {
            distance3 = dc;
            id3 = i;
        }
    }
    if (distance2 > -R) {
        const V3 D = position + row3(g.fn[id]) * distance; // closest point on face id
        bool edge2 = face_distance(g, id2, D) > 0.0;
        if (distance3 > -R && face_distance(g, id3, D) > 0.0) {
            const V3 E = position + row3(g.fn[id2]) * distance2;
            const bool edge3 = face_distance(g, id3, E) > 0.0;
            if (edge2) {
                if (edge3) {
                    if (id2 > id3) {
                        const unsigned t = id2;
                        id2 = id3;
                        id3 = t;
                    }
                    const unsigned index = (id < id2)   ? ((id3 - 2) * (id3 - 1) * id3 / 6 + (id2 - 1) * id2 / 2 + id)
                                           : (id < id3) ? ((id3 - 2) * (id3 - 1) * id3 / 6 + (id - 1) * id / 2 + id2)
                                                        : ((id - 2) * (id - 1) * id / 6 + (id3 - 1) * id3 / 2 + id2);
                    normal = position - row3(g.C[index]);
                    distance = sqrt(len2(normal));
                    if (distance <= R) {
                        normal = normal / (-distance);
                        return true;
                    }
                    if (distance == distance) return false;
                }
            } else {
                edge2 = true;
                distance2 = distance3;
                id2 = id3;
            }
        }
        if (edge2) {
            const unsigned index = (id > id2) ? ((id - 1) * id / 2 + id2) : ((id2 - 1) * id2 / 2 + id);
            const V3 AB = row3(g.AB[index]);
            const V3 AC = position - row3(g.A[index]);
            normal = AC - AB * dot(AC, AB);
            distance = sqrt(len2(normal));
            if (distance <= R) {
                normal = normal / (-distance);
                return true;
            }
            if (distance == distance) return false;
        }
    }
    normal = row3(g.fn[id]);
    return true;
}

// TriangleWall::updateVertexAndNormal (TriangleWall.cc:218-249) from the
// wall's current position and orientation; Vec3D::normalise divides by the
// square root of the squared length (Vector.cc:124-132).
__host__ __device__ inline void triangle_geometry(const dem_wall& w, WallGeom& g)
{
    const Q4 q = wall_q(w);
    const V3 wp = v3(w.position[0], w.position[1], w.position[2]);
    V3 v[3];
    for (int i = 0; i < 3; ++i) v[i] = quat_to_lab(q, row3(g.tvl[i])) + wp;
    V3 e[3] = {v[1] - v[0], v[2] - v[1], v[0] - v[2]};
    V3 fn = cross(e[0], e[1]);
    fn = fn / sqrt(len2(fn));
    for (int i = 0; i < 3; ++i) {
        V3 en = cross(e[i], fn);
        const double l = sqrt(len2(e[i]));
        e[i] = e[i] / l;
        en = en / sqrt(len2(en));
        g.tv[i][0] = v[i].x; g.tv[i][1] = v[i].y; g.tv[i][2] = v[i].z;
        g.te[i][0] = e[i].x; g.te[i][1] = e[i].y; g.te[i][2] = e[i].z;
        g.ten[i][0] = en.x; g.ten[i][1] = en.y; g.ten[i][2] = en.z;
        g.tel[i] = l;
    }
    g.tfn[0] = fn.x; g.tfn[1] = fn.y; g.tfn[2] = fn.z;
    for (int k = 0; k < 3; ++k) {
        g.tlo[k] = fmin(fmin(g.tv[0][k], g.tv[1][k]), g.tv[2][k]);
        g.thi[k] = fmax(fmax(g.tv[0][k], g.tv[1][k]), g.tv[2][k]);
    }
}

// TriangleWall::isInsideTriangle (TriangleWall.cc:251-262): the three
// area ratios are tested as written there, `1 > s > 0`, which C++ evaluates
// as (1 > s) > 0, i.e. s < 1.
__host__ __device__ __forceinline__ bool triangle_inside(const WallGeom& g, V3 p)
{
    const V3 v0 = row3(g.tv[0]), v1 = row3(g.tv[1]), v2 = row3(g.tv[2]);
    const V3 b0 = p - v0, b1 = p - v1, b2 = p - v2;
    const double s = sqrt(len2(cross(v1 - v0, v2 - v1)));
    const double s0 = sqrt(len2(cross(b0, b1))) / s;
    const double s1 = sqrt(len2(cross(b1, b2))) / s;
    const double s2 = sqrt(len2(cross(b2, b0))) / s;
    return s0 < 1 && s1 < 1 && s2 < 1;
}

// TriangleWall::getDistanceAndNormal (TriangleWall.cc:57-104): face contact
// if the particle projects inside the triangle, else the edge of largest
// in-plane distance or one of its vertices. R is the wall interaction radius.
__host__ __device__ __forceinline__ bool triangle_distance(const WallGeom& g, V3 x, double R, double& dist,
                                                           V3& normal)
{
    const V3 fn = row3(g.tfn);
    const double sd = dot(x - row3(g.tv[0]), fn);
    dist = fabs(sd);
    if (dist >= R) return false;
    // selected by value, not by a local array index (which would live on the stack)
    const V3 b0 = x - row3(g.tv[0]), b1 = x - row3(g.tv[1]), b2 = x - row3(g.tv[2]);
    const double e0 = dot(b0, row3(g.ten[0])), e1 = dot(b1, row3(g.ten[1])), e2 = dot(b2, row3(g.ten[2]));
    const int id = (e1 > e2) ? (e0 > e1 ? 0 : 1) : (e0 > e2 ? 0 : 2);
    const double eid = (id == 0) ? e0 : (id == 1) ? e1 : e2;
    if (eid > R) return false;
    const V3 proj = x - sd * fn;
    if (eid <= 0 && triangle_inside(g, proj)) {
        normal = (sd >= 0) ? -fn : fn;
        return true;
    }
    const V3 bid = (id == 0) ? b0 : (id == 1) ? b1 : b2;
    const V3 e = row3(g.te[id]);
    const double along = dot(bid, e);
    if (along < 0) {
        dist = sqrt(len2(bid));
        if (dist > R) return false;
        normal = bid / -dist;
    } else if (along > g.tel[id]) {
        const V3 bnext = (id == 0) ? b1 : (id == 1) ? b2 : b0; // vertex (id + 1) % 3
        dist = sqrt(len2(bnext));
        if (dist > R) return false;
        normal = bnext / -dist;
    } else {
        normal = e * along - bid;
        dist = sqrt(len2(normal));
        if (dist > R) return false;
        normal = normal / dist;
    }
    return true;
}

// TriangleWall::isFaceContact (TriangleWall.h:151-153): exact comparison
// with the face normal or its negative.
__host__ __device__ __forceinline__ bool triangle_face_contact(const WallGeom& g, V3 n)
{
    const V3 fn = row3(g.tfn);
    return (n.x == fn.x && n.y == fn.y && n.z == fn.z) || (n.x == -fn.x && n.y == -fn.y && n.z == -fn.z);
}

// BaseWall::getDistanceNormalOverlap for the supported wall types: signed
// distance of x from the wall and the wall's outward normal at the contact;
// false when x is not within R of the wall.
__host__ __device__ __forceinline__ bool wall_distance(const dem_wall& w, const WallGeom* geom, V3 x, double R,
                                                       double& dist, V3& normal)
{
    const Q4 q = wall_q(w);
    const V3 wp = v3(w.position[0], w.position[1], w.position[2]);
    if (w.type == DEM_WALL_INFINITE) {
        dist = quat_plane_distance(q, x, wp);
        if (dist >= R) return false;
        normal = quat_axis(q);
        return true;
    }
    if (w.type == DEM_WALL_AXISYMMETRIC) {
        const V3 po = x - wp;
        const V3 axis = quat_axis(q);
        const double a = dot(po, axis);
        V3 radial = po - a * axis;
        const double r = sqrt(len2(radial));
        V3 nrz;
        if (!intersection_distance(*geom, w.n_faces, v3(r, 0.0, a), R, dist, nrz)) return false;
        if (r != 0) radial = radial / r;
        normal = nrz.z * axis + nrz.x * radial;
        return true;
    }
    // DEM_WALL_INTERSECTION (triangle walls: triangle_distance, called by k_tri only)
    const V3 pb = quat_to_body(q, x - wp);
    V3 nb;
    if (!intersection_distance(*geom, w.n_faces, pb, R, dist, nb)) return false;
    normal = quat_to_lab(q, nb);
    return true;
}

// ---- host-side set-up --------------------------------------------------

// Quaternion::setOrientationViaNormal (Quaternion.cc:543-567), which first
// normalises the normal: the rotation taking (1, 0, 0) to the normal.
__host__ inline Q4 orientation_from_normal(V3 n)
{
    n = n / sqrt(len2(n));
    if (n.x <= -1 + 1e-14) return Q4{0.0, 0.0, 1.0, 0.0};
    const V3 half = V3{1.0 + n.x, 0.0 + n.y, 0.0 + n.z};
    Q4 q{half.x, 0.0, -half.z, half.y};
    const double l = sqrt(q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3);
    q.q0 /= l;
    q.q1 /= l;
    q.q2 /= l;
    q.q3 /= l;
    return q;
}

// The point where three planes {x : x . n_k = b_k} meet, by Cramer's rule
// with the cofactor order of IntersectionOfWalls::setPointsAndLines
// (IntersectionOfWalls.cc:365-389 for the edge point, with the edge
// direction as third plane and b = 0; :399-433 for a corner).
__host__ inline V3 three_plane_point(V3 a, V3 b, V3 c, double ba, double bb, double bc)
{
    const double invdet = 1.0 / (+a.x * (b.y * c.z - c.y * b.z) - a.y * (b.x * c.z - b.z * c.x) +
                                 a.z * (b.x * c.y - b.y * c.x));
    const V3 r{+(b.y * c.z - c.y * b.z) * ba - (a.y * c.z - a.z * c.y) * bb + (a.y * b.z - a.z * b.y) * bc,
               -(b.x * c.z - b.z * c.x) * ba + (a.x * c.z - a.z * c.x) * bb - (a.x * b.z - b.x * a.z) * bc,
               +(b.x * c.y - c.x * b.y) * ba - (a.x * c.y - c.x * a.y) * bb + (a.x * b.y - b.x * a.y) * bc};
    return r * invdet;
}

// Vec3D::cross (Vector.cc:164-167)
__host__ inline V3 cross_ref(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Faces are added one at a time, each followed by its edges with the earlier
// faces and its corners with every earlier pair (IntersectionOfWalls::addObject
// then setPointsAndLines).
__host__ inline void build_wall_geom(const dem_wall& w, WallGeom& g)
{
    std::memset(&g, 0, sizeof(g));
    if (w.type == DEM_WALL_TRIANGLE) { // TriangleWall::setVertices(A, B, C, position)
        const V3 wp = v3(w.position[0], w.position[1], w.position[2]);
        for (int i = 0; i < 3; ++i) {
            const V3 r = row3(w.faces[i]) - wp;
            g.tvl[i][0] = r.x; g.tvl[i][1] = r.y; g.tvl[i][2] = r.z;
        }
        triangle_geometry(w, g);
        return;
    }
    for (int n = 0; n < w.n_faces; ++n) {
        V3 nrm = row3(w.faces[n]);
        nrm = nrm / sqrt(len2(nrm)); // addObject normalises, setNormal normalises again
        const Q4 q = orientation_from_normal(nrm);
        g.fq[n][0] = q.q0; g.fq[n][1] = q.q1; g.fq[n][2] = q.q2; g.fq[n][3] = q.q3;
        for (int k = 0; k < 3; ++k) g.fp[n][k] = w.faces[n][3 + k];
        const V3 ax = quat_axis(q);
        g.fn[n][0] = ax.x; g.fn[n][1] = ax.y; g.fn[n][2] = ax.z;
        const V3 Nn = ax, Pn = row3(g.fp[n]);
        for (int m = 0; m < n; ++m) {
            const int id = (n - 1) * n / 2 + m;
            const V3 Nm = row3(g.fn[m]), Pm = row3(g.fp[m]);
            V3 AB = cross_ref(Nm, Nn);
            AB = AB / sqrt(len2(AB));
            const V3 A = three_plane_point(Nn, Nm, AB, dot(Pn, Nn), dot(Pm, Nm), 0.0);
            g.AB[id][0] = AB.x; g.AB[id][1] = AB.y; g.AB[id][2] = AB.z;
            g.A[id][0] = A.x; g.A[id][1] = A.y; g.A[id][2] = A.z;
        }
        for (int m = 0; m < n; ++m)
            for (int l = 0; l < m; ++l) {
                const int id = (n - 2) * (n - 1) * n / 6 + (m - 1) * m / 2 + l;
                const V3 Nm = row3(g.fn[m]), Pm = row3(g.fp[m]);
                const V3 Nl = row3(g.fn[l]), Pl = row3(g.fp[l]);
                const V3 C = three_plane_point(Nn, Nm, Nl, dot(Pn, Nn), dot(Pm, Nm), dot(Pl, Nl));
                g.C[id][0] = C.x; g.C[id][1] = C.y; g.C[id][2] = C.z;
            }
    }
}

} // namespace dem
