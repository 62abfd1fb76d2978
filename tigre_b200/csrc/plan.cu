// Plan creation: FP64 per-angle frames of the cone-beam geometry, uploaded
// once; error state; the stream-ordered scratch arena.
//
// The frame formulas are the reference's (they define the geometry and must
// agree with it); each block cites the function it restates:
//   Siddon frame      computeDeltas_Siddon, Common/CUDA/Siddon_projection.cu:666-763
//   rotations         rollPitchYaw, Common/CUDA/projection.cpp:18-35;
//                     eulerZYZ, Siddon_projection.cu:801-820
//   interpolated      computeDeltas + maxdistanceCuboid, ray_interpolated_projection.cu:632-768
//   backprojection    computeDeltasCube + eulerZYZT + rollPitchYawT,
//                     Common/CUDA/voxel_backprojection.cu:762-898
// The reference evaluates most of them in float; here everything is double.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "tigre_internal.h"

namespace tigre {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

namespace {
std::atomic<unsigned long long> g_launches{0};
}

void note_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// ---- library options (tigre_set_option) ----
namespace {
constexpr int kNumOptions = 8;
// defaults: SIDDON_KERNEL 0, BP_BOX 0, BP_KERNEL 0, HOST_CHUNK_VIEWS 0, HOST_STAGING -1, BP_SKIP_COPY -1,
// INTERP_TEXTURE 0
std::atomic<long long> g_options[kNumOptions] = {{0}, {0}, {0}, {0}, {0}, {-1}, {-1}, {0}};
}  // namespace

long long option(int key) {
    return (key > 0 && key < kNumOptions) ? g_options[key].load(std::memory_order_relaxed) : 0;
}

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return TIGRE_ERR_CUDA;
}

namespace {

struct Vec { double x, y, z; };

struct Rot3 {
    double m[3][3];
    Vec apply(const Vec& p) const {
        return {m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z, m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z,
                m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z};
    }
    Rot3 transposed() const {
        Rot3 t;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) t.m[i][j] = m[j][i];
        return t;
    }
};

// detector roll/pitch/yaw (projection.cpp:18-35)
Rot3 detector_rotation(double roll, double pitch, double yaw) {
    const double cr = std::cos(roll), sr = std::sin(roll), cp = std::cos(pitch), sp = std::sin(pitch);
    const double cy = std::cos(yaw), sy = std::sin(yaw);
    Rot3 r;
    r.m[0][0] = cr * cp; r.m[0][1] = cr * sp * sy - sr * cy; r.m[0][2] = cr * sp * cy + sr * sy;
    r.m[1][0] = sr * cp; r.m[1][1] = sr * sp * sy + cr * cy; r.m[1][2] = sr * sp * cy - cr * sy;
    r.m[2][0] = -sp;     r.m[2][1] = cp * sy;                r.m[2][2] = cp * cy;
    return r;
}

// ZYZ Euler rotation (Siddon_projection.cu:801-820); eulerZYZT of the
// backprojectors is the same matrix at negated angles.
Rot3 euler_zyz(double a, double t, double p) {
    const double ca = std::cos(a), sa = std::sin(a), ct = std::cos(t), st = std::sin(t);
    const double cp = std::cos(p), sp = std::sin(p);
    Rot3 r;
    r.m[0][0] = ca * ct * cp - sa * sp; r.m[0][1] = -ca * ct * sp - sa * cp; r.m[0][2] = ca * st;
    r.m[1][0] = sa * ct * cp + ca * sp; r.m[1][1] = -sa * ct * sp + ca * cp; r.m[1][2] = sa * st;
    r.m[2][0] = -st * cp;               r.m[2][1] = st * sp;                 r.m[2][2] = ct;
    return r;
}

// eulerZYZT (voxel_backprojection.cu:762-785): entries arranged with psi/alpha swapped
Rot3 euler_zyz_T(double a, double t, double p) {
    const double ca = std::cos(a), sa = std::sin(a), ct = std::cos(t), st = std::sin(t);
    const double cp = std::cos(p), sp = std::sin(p);
    Rot3 r;
    r.m[0][0] = cp * ct * ca - sp * sa; r.m[0][1] = -cp * ct * sa - sp * ca; r.m[0][2] = cp * st;
    r.m[1][0] = sp * ct * ca + cp * sa; r.m[1][1] = -sp * ct * sa + cp * ca; r.m[1][2] = sp * st;
    r.m[2][0] = -st * ca;               r.m[2][1] = st * sa;                 r.m[2][2] = ct;
    return r;
}

inline double at(const float* a, int i) { return a ? (double)a[i] : 0.0; }

}  // namespace

// Exact bounds for the cell-interval Siddon kernel, evaluated with the kernel's own FP64 ray
// setup for every view and detector column: within one column the z component of the ray
// is linear in the row, so its extremes are the first and the last row.
void cells_bounds(TigrePlan* plan) {
    const Dims& d = plan->d;
    double slope = 0.0, span = 0.0;
    for (const FrameSiddon& f : plan->h_siddon) {
        for (int u = 0; u < d.nU; ++u) {
            // the kernels' ray setup; in parallel beam each pixel has its own source
            const double sx = plan->parallel ? std::fma((double)u, f.du[0], f.s[0]) : f.s[0];
            const double sy = plan->parallel ? std::fma((double)u, f.du[1], f.s[1]) : f.s[1];
            double rx = std::fma((double)u, f.du[0], f.o[0]) - sx;
            double ry = std::fma((double)u, f.du[1], f.o[1]) - sy;
            if (std::fabs(rx) < 0.001) rx = 0.0;
            if (std::fabs(ry) < 0.001) ry = 0.0;
            double am = -1e300, aM = 1e300;
            bool miss = false;
            if (rx != 0.0) {
                const double i = 1.0 / rx, a0 = -sx * i, a1 = ((double)d.nX - sx) * i;
                am = std::fmax(am, std::fmin(a0, a1)); aM = std::fmin(aM, std::fmax(a0, a1));
            } else if (sx < 0.0 || sx > (double)d.nX) miss = true;
            if (ry != 0.0) {
                const double i = 1.0 / ry, a0 = -sy * i, a1 = ((double)d.nY - sy) * i;
                am = std::fmax(am, std::fmin(a0, a1)); aM = std::fmin(aM, std::fmax(a0, a1));
            } else if (sy < 0.0 || sy > (double)d.nY) miss = true;
            if (miss || !(am < aM)) continue;
            const double dom = std::max(std::fabs(rx), std::fabs(ry));
            for (int e = 0; e < 2; ++e) {
                const double pv = e ? 0.0 : (double)(d.nV - 1);
                const double sz = plan->parallel ? std::fma(pv, f.dv[2], std::fma((double)u, f.du[2], f.s[2])) : f.s[2];
                double rz = std::fma(pv, f.dv[2], std::fma((double)u, f.du[2], f.o[2])) - sz;
                if (std::fabs(rz) < 0.001) rz = 0.0;
                slope = std::max(slope, dom > 0.0 ? std::fabs(rz) / dom : 1e30);
                span = std::max(span, (aM - am) * std::fabs(rz));
            }
        }
    }
    plan->cells_slope_max = slope;
    plan->cells_zspan_max = span;
    // the exact slope also governs the one-crossing variant of the stepped column kernel
    plan->column_slope_max = std::max(plan->column_slope_max, slope);
    // one z crossing per xy cell at most (z change per cell < 1, with margin), and pads that
    // stay a modest multiple of the volume
    const double pad = std::ceil(span) + 3.0;
    const bool ok = slope < 0.9 && pad <= 2.0 * d.nZ + 256.0 && option(TIGRE_OPT_SIDDON_KERNEL) == 0;
    plan->cells_zpad = ok ? (int)pad : 0;
}

// Parallel-beam frames.  Every pixel has its own source: source(u, v) = s + u du + v dv.
//  * Siddon (computeDeltas_Siddon_parallel, Siddon_projection_parallel.cu:388-480): pixel
//    (0,0) on the plane x = DSO; rotation about z by alpha only; the detector offset moves
//    the detector points, not the source.
//  * interpolated (computeDeltas_parallel, ray_interpolated_projection_parallel.cu:309-400):
//    full ZYZ Euler rotation, detector offset applied twice (:341-356), voxel centres at
//    integers; sample cap with dVoxelX (:175-176).
//  * backprojection (computeDeltasCubeParallel, voxel_backprojection_parallel.cu:510-585, the
//    steps of the cone frame): the voxel projects orthographically, u = y - COR/dDetecU + nU/2
//    and v = z + nV/2 in texture coordinates, weight 1 (:221-250).  This is encoded in the cone
//    FDK frame: the depth row is made constant 1 (o.x = dx.x = dy.x = dz.x = 0, s.x = -1), the
//    numerator DSO - DSD - s.x is 1 (DSO = DSD = 1), s.y = s.z = 0 and the FDK weight's
//    sin/cos are 0, so t = 1 and the weight is 1 exactly.
void parallel_frames(const TigreGeometry* g, const Dims& d, int i, double al, double th, double ps, TigrePlan* plan) {
    const double dso = g->DSO[i], dsd = g->DSD[i];
    const double offx = at(g->offOrigX, i), offy = at(g->offOrigY, i), offz = at(g->offOrigZ, i);
    const double offu = at(g->offDetecU, i), offv = at(g->offDetecV, i);
    const double cor = at(g->COR, i);
    const Rot3 rd = detector_rotation(at(g->dRoll, i), at(g->dPitch, i), at(g->dYaw, i));
    const double y0 = d.dDU * (-(double)d.nU / 2.0 + 0.5), z0 = d.dDV * ((double)d.nV / 2.0 - 0.5);
    const double corx = -cor * std::sin(al) / d.dVX, cory = cor * std::cos(al) / d.dVY;
    auto frame = [&](const Rot3& rot, double offmul, double centre, double o3[3], double du3[3], double dv3[3],
                     double s3[3]) {
        Vec P{0.0, y0, z0}, Pu{0.0, y0 + d.dDU, z0}, Pv{0.0, y0, z0 - d.dDV}, S{0.0, y0, z0};
        for (Vec* q : {&P, &Pu, &Pv}) {
            *q = rd.apply(*q);
            q->x -= (dsd - dso);
            q->y += offmul * offu;
            q->z += offmul * offv;
        }
        S = rd.apply(S);
        S.x += dso;
        for (Vec* q : {&P, &Pu, &Pv, &S}) {
            *q = rot.apply(*q);
            q->x = (q->x - offx + d.sVX / 2 - centre * d.dVX) / d.dVX + corx;
            q->y = (q->y - offy + d.sVY / 2 - centre * d.dVY) / d.dVY + cory;
            q->z = (q->z - offz + d.sVZ / 2 - centre * d.dVZ) / d.dVZ;
        }
        o3[0] = P.x; o3[1] = P.y; o3[2] = P.z;
        du3[0] = Pu.x - P.x; du3[1] = Pu.y - P.y; du3[2] = Pu.z - P.z;
        dv3[0] = Pv.x - P.x; dv3[1] = Pv.y - P.y; dv3[2] = Pv.z - P.z;
        s3[0] = S.x; s3[1] = S.y; s3[2] = S.z;
    };
    FrameSiddon& fs = plan->h_siddon[i];
    frame(euler_zyz(al, 0.0, 0.0), 1.0, 0.0, fs.o, fs.du, fs.dv, fs.s);
    fs.layout = std::fabs(fs.du[1]) >= std::fabs(fs.du[0]) ? 1 : 0;
    fs.pad_ = 0;
    FrameInterp& fi = plan->h_interp[i];
    frame(euler_zyz(al, th, ps), 2.0, 0.5, fi.o, fi.du, fi.dv, fi.s);
    fi.layout = std::fabs(fi.du[1]) >= std::fabs(fi.du[0]) ? 1 : 0;
    fi.pad_ = 0;
    {
        // maxdistanceCuboid as for cone beam; cap with dVoxelX
        const double mx = (double)(d.nX / 2) + std::fabs(offx) / d.dVX;
        const double my = (double)(d.nY / 2) + std::fabs(offy) / d.dVY;
        const double mz = (double)(d.nZ / 2) + std::fabs(offz) / d.dVZ;
        const double a = dso / d.dVX, b = dso / d.dVY;
        double md;
        if (th == 0.0 && ps == 0.0) {
            const double sa = std::sin(al), ca = std::cos(al);
            md = a * b / std::sqrt(a * a * sa * sa + b * b * ca * ca) - std::sqrt(mx * mx + my * my);
        } else {
            md = dso / std::max(std::max(d.dVX, d.dVY), d.dVZ) - std::sqrt(mx * mx + my * my + mz * mz);
        }
        const double crop = std::floor(std::max(md, 0.0));
        fi.first_sample = std::floor(crop / d.accuracy);
        fi.cap = (2.0 * dso / d.dVX + crop) / d.accuracy;
    }
    // backprojection frame: the cone frame's steps, then the orthographic encoding
    const Rot3 rt = euler_zyz_T(-al, -th, -ps);
    const Rot3 rdt = rd.transposed();
    Vec Q{-(d.sVX / 2 - d.dVX / 2) + offx, -(d.sVY / 2 - d.dVY / 2) + offy, -(d.sVZ / 2 - d.dVZ / 2) + offz};
    Vec pts[4] = {Q, {Q.x + d.dVX, Q.y, Q.z}, {Q.x, Q.y + d.dVY, Q.z}, {Q.x, Q.y, Q.z + d.dVZ}};
    const double off = dsd - dso;
    for (Vec& q : pts) {
        q = rt.apply(q);
        q.z -= offv; q.y -= offu;
        q.x += off;
        q = rdt.apply(q);
        q.x -= off;
        q.z /= d.dDV; q.y /= d.dDU;
    }
    FrameBP& fb = plan->h_bp[i];
    fb.o[0] = 0.0; fb.o[1] = pts[0].y; fb.o[2] = pts[0].z;
    fb.dx[0] = 0.0; fb.dx[1] = pts[1].y - pts[0].y; fb.dx[2] = pts[1].z - pts[0].z;
    fb.dy[0] = 0.0; fb.dy[1] = pts[2].y - pts[0].y; fb.dy[2] = pts[2].z - pts[0].z;
    fb.dz[0] = 0.0; fb.dz[1] = pts[3].y - pts[0].y; fb.dz[2] = pts[3].z - pts[0].z;
    fb.s[0] = -1.0; fb.s[1] = 0.0; fb.s[2] = 0.0;
    fb.sina = 0.f; fb.cosa = 0.f;
    fb.cor = (float)cor; fb.dsd = 1.f; fb.dso = 1.f;
    fb.offx = (float)offx; fb.offy = (float)offy; fb.offz = (float)offz;
    fb.offu = (float)offu; fb.offv = (float)offv;
}

// Shared-memory wavefronts of the staged backprojector's four bilinear taps for a patch of
// es-byte texels and row pitch BU texels, estimated on sample blocks, views and slices with the kernel's own
// thread layout (a warp = 8 x 4 voxel columns) and patch origin rule.  A warp load costs as
// many wavefronts as the largest number of distinct words that fall in one bank.
double bp_bank_cost(const TigrePlan* plan, int BU, int es, int bx, int bz) {
    const Dims& d = plan->d;
    const int na = (int)plan->h_bpk.size();
    const int vstep_views = std::max(1, na / 24);
    const int nbx = (d.nX + bx - 1) / bx, nby = (d.nY + bx - 1) / bx, nbz = (d.nZ + bz - 1) / bz;
    const int sbx[3] = {0, nbx / 2, nbx - 1}, sby[3] = {0, nby / 2, nby - 1}, sbz[2] = {0, nbz / 2};
    const int warps[2] = {0, 5};
    const int slices[4] = {0, bz / 3, (2 * bz) / 3, bz - 1};
    double cost = 0.0;
    for (int a = 0; a < na; a += vstep_views) {
        const FrameBPK& k = plan->h_bpk[a];
        auto proj = [&](double x, double y, double z, double& u, double& v) {
            const double vx = k.b[0] + x * k.dx[0] + y * k.dy[0] + z * k.dz[0];
            const double vy = k.b[1] + x * k.dx[1] + y * k.dy[1] + z * k.dz[1];
            const double vz = k.b[2] + x * k.dx[2] + y * k.dy[2] + z * k.dz[2];
            const double t = (double)k.tnum / vx;
            u = vy * t + k.cu - 0.5;
            v = vz * t + k.cv - 0.5;
        };
        for (int ix : sbx)
            for (int iy : sby)
                for (int iz : sbz) {
                    const int x0 = ix * bx, y0 = iy * bx, z0 = iz * bz;
                    double umin = 1e300, vmin = 1e300;
                    for (int c = 0; c < 8; ++c) {
                        double u, v;
                        proj(std::min(x0 + ((c & 1) ? bx - 1 : 0), d.nX - 1), std::min(y0 + ((c & 2) ? bx - 1 : 0), d.nY - 1),
                             std::min(z0 + ((c & 4) ? bz - 1 : 0), d.nZ - 1), u, v);
                        umin = std::min(umin, u);
                        vmin = std::min(vmin, v);
                    }
                    if (!std::isfinite(umin) || !std::isfinite(vmin)) continue;
                    int u0 = (int)std::floor(umin) - 1;
                    const int al = 16 / es;   // TMA: the patch origin's x is 16-byte aligned
                    u0 = u0 >= 0 ? (u0 / al) * al : -(((-u0) + al - 1) / al) * al;
                    const int v0 = (int)std::floor(vmin) - 1;
                    for (int w : warps)
                        for (int ks : slices) {
                            long words[4][32];
                            for (int ln = 0; ln < 32; ++ln) {
                                const int x = x0 + (w & 1) * 8 + (ln & 7), y = y0 + (w >> 1) * 4 + (ln >> 3);
                                double u, v;
                                proj(std::min(x, d.nX - 1), std::min(y, d.nY - 1), std::min(z0 + ks, d.nZ - 1), u, v);
                                const long iu = (long)std::floor(u - u0), iv = (long)std::floor(v - v0);
                                const long base = iv * BU + iu;
                                words[0][ln] = base * es / 4; words[1][ln] = (base + 1) * es / 4;
                                words[2][ln] = (base + BU) * es / 4; words[3][ln] = (base + BU + 1) * es / 4;
                            }
                            for (auto& tap : words) {
                                int per_bank[32] = {0};
                                std::sort(tap, tap + 32);
                                for (int ln = 0; ln < 32; ++ln)
                                    if (ln == 0 || tap[ln] != tap[ln - 1]) ++per_bank[((tap[ln] % 32) + 32) % 32];
                                cost += *std::max_element(per_bank, per_bank + 32);
                            }
                        }
                }
    }
    return cost;
}

int compute_frames(const TigreGeometry* g, const float* angles, int nangles, TigrePlan* plan) {
    TIGRE_CHECK(g != nullptr && angles != nullptr, "null geometry or angles");
    TIGRE_CHECK(nangles > 0, "nangles must be positive");
    TIGRE_CHECK(g->nVoxelX > 0 && g->nVoxelY > 0 && g->nVoxelZ > 0, "nVoxel must be positive");
    TIGRE_CHECK(g->nDetecU > 0 && g->nDetecV > 0, "nDetector must be positive");
    TIGRE_CHECK(g->DSO && g->DSD, "DSO/DSD arrays are required");
    TIGRE_CHECK((double)g->nVoxelX * g->nVoxelY * g->nVoxelZ < 2147483647.0 * 0.99,
                "volume larger than 2^31 voxels is not supported");
    Dims& d = plan->d;
    d.nX = g->nVoxelX; d.nY = g->nVoxelY; d.nZ = g->nVoxelZ;
    d.nU = g->nDetecU; d.nV = g->nDetecV; d.nA = nangles;
    d.sVX = g->sVoxelX; d.sVY = g->sVoxelY; d.sVZ = g->sVoxelZ;
    d.dVX = g->dVoxelX; d.dVY = g->dVoxelY; d.dVZ = g->dVoxelZ;
    d.sDU = g->sDetecU; d.sDV = g->sDetecV; d.dDU = g->dDetecU; d.dDV = g->dDetecV;
    d.accuracy = g->accuracy;
    TIGRE_CHECK(d.dVX > 0 && d.dVY > 0 && d.dVZ > 0 && d.dDU > 0 && d.dDV > 0, "voxel/pixel sizes must be positive");
    TIGRE_CHECK(d.accuracy > 0, "accuracy must be positive");

    plan->h_siddon.resize(nangles);
    plan->h_interp.resize(nangles);
    plan->h_bp.resize(nangles);
    bool axial = true, columns = true;
    for (int i = 0; i < nangles; ++i) {
        const double al = angles[3 * i], th = angles[3 * i + 1], ps = angles[3 * i + 2];
        const double dso = g->DSO[i], dsd = g->DSD[i];
        const double offx = at(g->offOrigX, i), offy = at(g->offOrigY, i), offz = at(g->offOrigZ, i);
        const double offu = at(g->offDetecU, i), offv = at(g->offDetecV, i);
        const double cor = at(g->COR, i);
        const Rot3 rd = detector_rotation(at(g->dRoll, i), at(g->dPitch, i), at(g->dYaw, i));
        const Rot3 re = euler_zyz(al, th, ps);

        if (plan->parallel) {
            parallel_frames(g, d, i, al, th, ps, plan);
            if (plan->h_siddon[i].dv[0] != 0.0 || plan->h_siddon[i].dv[1] != 0.0) columns = false;
            const FrameBP& fb = plan->h_bp[i];
            if (std::fabs(fb.dz[0]) > 1e-12 * d.dVZ || std::fabs(fb.dz[1]) > 1e-12 * d.dVZ) axial = false;
            continue;
        }
        // ---- Siddon frame (computeDeltas_Siddon) ----
        Vec S{dso, 0.0, 0.0};
        Vec P{0.0, d.dDU * (-(double)d.nU / 2.0 + 0.5), d.dDV * ((double)d.nV / 2.0 - 0.5)};
        Vec Pu{0.0, d.dDU, 0.0}, Pv{0.0, 0.0, -d.dDV};
        P = rd.apply(P); Pu = rd.apply(Pu); Pv = rd.apply(Pv);
        P.x -= (dsd - dso);
        P.y += offu; P.z += offv;
        P = re.apply(P); Pu = re.apply(Pu); Pv = re.apply(Pv); S = re.apply(S);
        const double cx = -offx + d.sVX / 2, cy = -offy + d.sVY / 2, cz = -offz + d.sVZ / 2;
        P = {(P.x + cx) / d.dVX, (P.y + cy) / d.dVY, (P.z + cz) / d.dVZ};
        S = {(S.x + cx) / d.dVX, (S.y + cy) / d.dVY, (S.z + cz) / d.dVZ};
        Pu = {Pu.x / d.dVX, Pu.y / d.dVY, Pu.z / d.dVZ};
        Pv = {Pv.x / d.dVX, Pv.y / d.dVY, Pv.z / d.dVZ};
        const double corx = -cor * std::sin(al) / d.dVX, cory = cor * std::cos(al) / d.dVY;
        P.x += corx; P.y += cory; S.x += corx; S.y += cory;
        FrameSiddon& fs = plan->h_siddon[i];
        fs.o[0] = P.x; fs.o[1] = P.y; fs.o[2] = P.z;
        fs.du[0] = Pu.x; fs.du[1] = Pu.y; fs.du[2] = Pu.z;
        fs.dv[0] = Pv.x; fs.dv[1] = Pv.y; fs.dv[2] = Pv.z;
        fs.s[0] = S.x; fs.s[1] = S.y; fs.s[2] = S.z;
        // neighbouring detector columns move mostly along y -> y-fastest working copy
        fs.layout = std::fabs(Pu.y) >= std::fabs(Pu.x) ? 1 : 0;
        fs.pad_ = 0;
        if (Pv.x != 0.0 || Pv.y != 0.0) columns = false;
        // steepest ray of this view: bounds the z crossings per xy cell.  |rz| is largest at
        // the first or last row; over u the ratio is sampled at 65 columns (and the threshold
        // used against it keeps a factor-2 margin)
        for (int cu = 0; cu <= 64; ++cu)
            for (int cv = 0; cv < 2; ++cv) {
                const double uu = (d.nU - 1) * (cu / 64.0), vv = cv ? d.nV - 1 : 0;
                const double rx = P.x + uu * Pu.x + vv * Pv.x - S.x, ry = P.y + uu * Pu.y + vv * Pv.y - S.y;
                const double rz = P.z + uu * Pu.z + vv * Pv.z - S.z;
                const double dom = std::max(std::fabs(rx), std::fabs(ry));
                plan->column_slope_max = std::max(plan->column_slope_max, dom > 0 ? std::fabs(rz) / dom : 1e30);
            }

        // ---- interpolated frame: voxel centres at integers (computeDeltas) ----
        FrameInterp& fi = plan->h_interp[i];
        for (int k = 0; k < 3; ++k) {
            fi.o[k] = fs.o[k] - 0.5; fi.du[k] = fs.du[k]; fi.dv[k] = fs.dv[k]; fi.s[k] = fs.s[k] - 0.5;
        }
        fi.layout = fs.layout;
        fi.pad_ = 0;
        {
            // maxdistanceCuboid: note the C integer division nVoxel/2 of the reference
            const double mx = (double)(d.nX / 2) + std::fabs(offx) / d.dVX;
            const double my = (double)(d.nY / 2) + std::fabs(offy) / d.dVY;
            const double mz = (double)(d.nZ / 2) + std::fabs(offz) / d.dVZ;
            const double a = dso / d.dVX, b = dso / d.dVY;
            double md;
            if (th == 0.0 && ps == 0.0) {
                const double sa = std::sin(al), ca = std::cos(al);
                md = a * b / std::sqrt(a * a * sa * sa + b * b * ca * ca) - std::sqrt(mx * mx + my * my);
            } else {
                md = dso / std::max(std::max(d.dVX, d.dVY), d.dVZ) - std::sqrt(mx * mx + my * my + mz * mz);
            }
            const double crop = std::floor(std::max(md, 0.0));
            fi.first_sample = std::floor(crop / d.accuracy);
            // the reference selects the spherical cap per launch of 9 angles
            const int b0 = (i / 9) * 9, b1 = std::min(b0 + 9, nangles);
            double sph = 0.0;
            for (int k = b0; k < b1; ++k) sph += std::fabs(angles[3 * k + 1]) + std::fabs(angles[3 * k + 2]);
            const double dmin = sph != 0.0 ? std::min(std::min(d.dVX, d.dVY), d.dVZ) : std::min(d.dVX, d.dVY);
            fi.cap = (2.0 * dso / dmin + crop) / d.accuracy;
        }

        // ---- backprojection frame (computeDeltasCube, angles negated) ----
        {
            const Rot3 rt = euler_zyz_T(-al, -th, -ps);
            const Rot3 rdt = detector_rotation(at(g->dRoll, i), at(g->dPitch, i), at(g->dYaw, i)).transposed();
            Vec Q{-(d.sVX / 2 - d.dVX / 2) + offx, -(d.sVY / 2 - d.dVY / 2) + offy, -(d.sVZ / 2 - d.dVZ / 2) + offz};
            Vec pts[4] = {Q, {Q.x + d.dVX, Q.y, Q.z}, {Q.x, Q.y + d.dVY, Q.z}, {Q.x, Q.y, Q.z + d.dVZ}};
            const double off = dsd - dso;
            for (Vec& p : pts) {
                p = rt.apply(p);
                p.z -= offv; p.y -= offu;
                p.x += off;
                p = rdt.apply(p);
                p.x -= off;
                p.z /= d.dDV; p.y /= d.dDU;
            }
            Vec src{dsd, -offu, -offv};
            src = rdt.apply(src);
            src.x -= off;
            src.z /= d.dDV; src.y /= d.dDU;
            FrameBP& fb = plan->h_bp[i];
            fb.o[0] = pts[0].x; fb.o[1] = pts[0].y; fb.o[2] = pts[0].z;
            const Vec* q = pts;
            fb.dx[0] = q[1].x - q[0].x; fb.dx[1] = q[1].y - q[0].y; fb.dx[2] = q[1].z - q[0].z;
            fb.dy[0] = q[2].x - q[0].x; fb.dy[1] = q[2].y - q[0].y; fb.dy[2] = q[2].z - q[0].z;
            fb.dz[0] = q[3].x - q[0].x; fb.dz[1] = q[3].y - q[0].y; fb.dz[2] = q[3].z - q[0].z;
            fb.s[0] = src.x; fb.s[1] = src.y; fb.s[2] = src.z;
            fb.sina = (float)std::sin(-al);
            fb.cosa = (float)std::cos(-al);
            fb.cor = (float)cor; fb.dsd = (float)dsd; fb.dso = (float)dso;
            fb.offx = (float)offx; fb.offy = (float)offy; fb.offz = (float)offz;
            fb.offu = (float)offu; fb.offv = (float)offv;
            if (std::fabs(fb.dz[0]) > 1e-12 * d.dVZ || std::fabs(fb.dz[1]) > 1e-12 * d.dVZ) axial = false;
        }
    }
    plan->axial = axial;
    plan->columns = columns && option(TIGRE_OPT_SIDDON_KERNEL) != 2;
    if (plan->columns) cells_bounds(plan);

    // ---- staged backprojector constants and patch box ----
    plan->h_bpk.resize(nangles);
    double ext_u = 0.0, ext_v = 0.0;
    const int bx = kBpTile, bz = kBpSlices;
    for (int i = 0; i < nangles; ++i) {
        const FrameBP& f = plan->h_bp[i];
        FrameBPK& k = plan->h_bpk[i];
        for (int c = 0; c < 3; ++c) { k.dx[c] = f.dx[c]; k.dy[c] = f.dy[c]; k.dz[c] = f.dz[c]; }
        k.b[0] = f.o[0] - f.s[0];
        k.b[1] = f.o[1] - (double)f.cor / d.dDU - f.s[1];
        k.b[2] = f.o[2] - f.s[2];
        k.tnum = (float)((double)f.dso - (double)f.dsd - f.s[0]);
        k.cu = (float)(f.s[1] + d.nU * 0.5);
        k.cv = (float)(f.s[2] + d.nV * 0.5);
        const double sina = f.sina, cosa = f.cosa;
        k.w0 = (float)(f.dso + (-(d.sVY - d.dVY) * 0.5 + f.offy + f.cor) * sina - (-(d.sVX - d.dVX) * 0.5 + f.offx) * cosa);
        k.wx = (float)(-d.dVX * cosa);
        k.wy = (float)(d.dVY * sina);
        k.dso = f.dso;
        k.dsd = f.dsd;
        k.rsx = (float)(f.dso * cosa);
        k.rsy = (float)(-f.dso * sina);
        const double dax = -((double)f.dsd - (double)f.dso);
        k.daxc = (float)(dax * cosa);
        k.daxs = (float)(dax * sina);
        k.sina = f.sina;
        k.cosa = f.cosa;
        k.du0 = (float)((-d.sDU + d.dDU) * 0.5 + f.offu);
        k.ddu = (float)d.dDU;
        k.dzc = (float)((-d.sDV + d.dDV) * 0.5 + f.offv);
        k.ddv = (float)d.dDV;
        k.rv0x = (float)(-d.sVX / 2 + d.dVX / 2 + f.offx);
        k.rv0y = (float)(-d.sVY / 2 + d.dVY / 2 + f.offy);
        k.rv0z = (float)(-d.sVZ / 2 + d.dVZ / 2 + f.offz);
        k.dvx = (float)d.dVX;
        k.dvy = (float)d.dVY;
        // footprint of sample blocks (first / middle / last along each axis) for this view
        const int nbx = (d.nX + bx - 1) / bx, nby = (d.nY + bx - 1) / bx, nbz = (d.nZ + bz - 1) / bz;
        const int sx[3] = {0, nbx / 2, nbx - 1}, sy[3] = {0, nby / 2, nby - 1}, sz[3] = {0, nbz / 2, nbz - 1};
        for (int ix = 0; ix < 3; ++ix)
            for (int iy = 0; iy < 3; ++iy)
                for (int iz = 0; iz < 3; ++iz) {
                    double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
                    for (int c = 0; c < 8; ++c) {
                        const double x = std::min(sx[ix] * bx + ((c & 1) ? bx - 1 : 0), d.nX - 1);
                        const double y = std::min(sy[iy] * bx + ((c & 2) ? bx - 1 : 0), d.nY - 1);
                        const double z = std::min(sz[iz] * bz + ((c & 4) ? bz - 1 : 0), d.nZ - 1);
                        const double vx = k.b[0] + x * k.dx[0] + y * k.dy[0] + z * k.dz[0];
                        const double vy = k.b[1] + x * k.dx[1] + y * k.dy[1] + z * k.dz[1];
                        const double vz = k.b[2] + x * k.dx[2] + y * k.dy[2] + z * k.dz[2];
                        const double t = (double)k.tnum / vx;
                        const double u = vy * t, v = vz * t;
                        umin = std::min(umin, u); umax = std::max(umax, u);
                        vmin = std::min(vmin, v); vmax = std::max(vmax, v);
                    }
                    ext_u = std::max(ext_u, umax - umin);
                    ext_v = std::max(ext_v, vmax - vmin);
                }
    }
    {
        // Patch box.  The TMA box's row must be a multiple of 16 bytes: 4 floats, 8 halves.
        const int need = (int)std::ceil(ext_u) + 13;
        int BV = (int)std::ceil(ext_v) + 6;
        if (BV < 4) BV = 4;
        // float rows: the pitch (mod 32 words) with the fewest estimated shared-memory wavefronts
        // among those whose double buffer fits the 96 KB budget
        const int base = (std::max(need, 4) + 3) / 4 * 4;
        int BU = base;
        while (BU % 8 != 4) BU += 4;
        double best = -1.0;
        for (int r = 0; r < 32; r += 4) {
            int bu = base;
            while (bu % 32 != r) bu += 4;
            if (bu > 256 || 2.0 * bu * BV * 4 > 96.0 * 1024) continue;
            const double c = bp_bank_cost(plan, bu, 4, bx, bz);
            if (best < 0.0 || c < best || (c == best && bu < BU)) { best = c; BU = bu; }
        }
        // 16-bit rows: the same choice over pitches = 0..56 (mod 64) halves
        const int base16 = (std::max(need, 8) + 7) / 8 * 8;
        int BU16 = base16;
        while (BU16 % 16 != 8) BU16 += 8;
        best = -1.0;
        for (int r = 0; r < 64; r += 8) {
            int bu = base16;
            while (bu % 64 != r) bu += 8;
            if (bu > 256 || 2.0 * bu * BV * 2 > 96.0 * 1024) continue;
            const double c = bp_bank_cost(plan, bu, 2, bx, bz);
            if (best < 0.0 || c < best || (c == best && bu < BU16)) { best = c; BU16 = bu; }
        }
        if (const long long box = option(TIGRE_OPT_BP_BOX)) {   // forced box (tests of the fallback path)
            const int bu = (int)((box >> 16) & 0xffff), bv = (int)(box & 0xffff);
            if (bu > 0 && bv > 0) {
                BU = (bu + 3) / 4 * 4;
                BU16 = (bu + 7) / 8 * 8;
                BV = bv;
            }
        }
        const bool ok = std::isfinite(ext_u) && std::isfinite(ext_v) && BU <= 256 && BU16 <= 256 && BV <= 256 &&
                        2.0 * BU * BV * 4 <= 96.0 * 1024 && option(TIGRE_OPT_BP_KERNEL) == 0;
        plan->bp_box_u = ok ? BU : 0;
        plan->bp_box_u16 = ok ? BU16 : 0;
        plan->bp_box_v = ok ? BV : 0;
    }
    return TIGRE_SUCCESS;
}

void* plan_scratch(TigrePlan* plan, size_t bytes, cudaStream_t st, int* rc) {
    *rc = TIGRE_SUCCESS;
    if (bytes <= plan->scratch_bytes) return plan->scratch;
    if (plan->scratch) {
        cudaError_t e = cudaFreeAsync(plan->scratch, st);
        if (e != cudaSuccess) { *rc = cuda_fail(e, "cudaFreeAsync(scratch)"); return nullptr; }
        plan->scratch = nullptr;
        plan->scratch_bytes = 0;
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess) { *rc = cuda_fail(e, "cudaMallocAsync(scratch)"); return nullptr; }
    plan->scratch = p;
    plan->scratch_bytes = bytes;
    return p;
}

}  // namespace tigre

using namespace tigre;

extern "C" {

const char* tigre_last_error(void) { return g_last_error.c_str(); }

int tigre_version(void) { return 101; }

long long tigre_set_option(int key, long long value) {
    if (key <= 0 || key >= kNumOptions) {
        fail(TIGRE_ERR_BAD_ASSERT, "unknown option " + std::to_string(key));
        return -1;
    }
    return g_options[key].exchange(value, std::memory_order_relaxed);
}

long long tigre_get_option(int key) {
    if (key <= 0 || key >= kNumOptions) {
        fail(TIGRE_ERR_BAD_ASSERT, "unknown option " + std::to_string(key));
        return -1;
    }
    return g_options[key].load(std::memory_order_relaxed);
}
unsigned long long tigre_launch_count(void) { return tigre::g_launches.load(std::memory_order_relaxed); }

int tigre_plan_create(const TigreGeometry* geo, const float* angles, int nangles, int device, TigrePlan** out) {
    return tigre_plan_create_ex(geo, angles, nangles, device, 0, out);
}

int tigre_plan_create_ex(const TigreGeometry* geo, const float* angles, int nangles, int device, int flags,
                         TigrePlan** out) {
    if (!out) return fail(TIGRE_ERR_BAD_ASSERT, "null output plan pointer");
    *out = nullptr;
    if (flags & ~TIGRE_PLAN_PARALLEL) return fail(TIGRE_ERR_BAD_ASSERT, "unknown plan flags");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(TIGRE_ERR_NO_CAPABLE_DEVICES, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(TIGRE_ERR_BAD_ASSERT, "device id out of range");
    TigrePlan* p = new TigrePlan();
    p->device = device;
    p->parallel = (flags & TIGRE_PLAN_PARALLEL) != 0;
    int rc = compute_frames(geo, angles, nangles, p);
    if (rc) { delete p; return rc; }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    const size_t ns = sizeof(FrameSiddon) * nangles, ni = sizeof(FrameInterp) * nangles, nb = sizeof(FrameBP) * nangles;
    const size_t nk = sizeof(FrameBPK) * nangles;
    e = cudaMalloc(&p->d_siddon, ns);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_interp, ni);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_bpk, nk);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(p->d_bpk, p->h_bpk.data(), nk, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_bp, nb);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_siddon, p->h_siddon.data(), ns, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_interp, p->h_interp.data(), ni, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->d_bp, p->h_bp.data(), nb, cudaMemcpyHostToDevice);
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        tigre_plan_destroy(p);
        return cuda_fail(e, "plan upload");
    }
    *out = p;
    return TIGRE_SUCCESS;
}

void tigre_plan_destroy(TigrePlan* p) {
    if (!p) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    if (p->scratch) { cudaDeviceSynchronize(); cudaFree(p->scratch); }
    cudaFree(p->d_siddon);
    cudaFree(p->d_interp);
    cudaFree(p->d_bp);
    cudaFree(p->d_bpk);
    cudaFree(p->d_status);
    if (p->tex_obj) cudaDestroyTextureObject((cudaTextureObject_t)p->tex_obj);
    if (p->tex_array) cudaFreeArray(p->tex_array);
    cudaSetDevice(prev);
    delete p;
}

long long tigre_plan_scratch_bytes(const TigrePlan* p) { return p ? (long long)p->scratch_bytes : 0; }

int tigre_plan_status(TigrePlan* p, int reset) {
    if (!p) return -1;
    int prev = 0, v = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    cudaDeviceSynchronize();
    cudaMemcpy(&v, p->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (reset) cudaMemset(p->d_status, 0, sizeof(int));
    cudaSetDevice(prev);
    return v;
}

}  // extern "C"
