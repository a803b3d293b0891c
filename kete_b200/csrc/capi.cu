// capi.cpp -- the extern "C" boundary: DAF/SPK ingest, device residency of the ephemeris,
// argument checking, host<->device staging and kernel dispatch.
//
// The ephemeris side restates DafFile::from_buffer / try_load_segments
// (src/kete_core/src/spice/daf.rs:148-262), SpkSegment / SpkSegmentType2 construction
// (spice/spk_segments.rs:105-135,379-397) and SpkCollection::load_file (spice/spk.rs:307-329).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kete_b200.h"
#include "common.cuh"
#include "ephem.cuh"
#include "flux.cuh"
#include "fov_args.h"
#include "internal.h"

namespace kb {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return 0;
    return set_error(KETE_B200_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------------------------------
// GravParams table (src/kete_core/src/constants/gravity.rs:43-148): PLANETS = first 10.
// ------------------------------------------------------------------------------------------
struct GravEntry {
    int64_t id;
    double mass_ratio, radius;
    int kind;
};
static const GravEntry MASSES[15] = {
    {10, 1.0, 0.004654758765894654, FK_SUN},
    {1, 1.66012082548908e-07, 1.63139354095098e-05, FK_PLAIN},
    {2, 2.44783828779694e-06, 4.04537843465442e-05, FK_PLAIN},
    {399, 3.00348961546514e-06, 4.33036684926559e-05, FK_EARTH},
    {301, 3.69430335010988e-08, 1.16138016662292e-05, FK_PLAIN},
    {4, 3.22715608291416e-07, 2.27021279387769e-05, FK_PLAIN},
    {5, 0.0009547919099414246, 0.00047789450254521576, FK_JUPITER},
    {6, 0.00028588567002459455, 0.0004028666966848747, FK_PLAIN},
    {7, 4.36624961322212e-05, 0.0001708513622580592, FK_PLAIN},
    {8, 5.15138377265457e-05, 0.0001655371154958558, FK_PLAIN},
    {20000001, 4.7191659919436e-10, 6.276827e-6, FK_PLAIN},
    {20000002, 1.0259143964958e-10, 3.415824e-6, FK_PLAIN},
    {20000004, 1.3026452498655e-10, 3.512082e-6, FK_PLAIN},
    {20000010, 4.3953391300849e-11, 2.894426e-6, FK_PLAIN},
    {20000704, 1.911e-11, 2.219283e-6, FK_PLAIN},
};
constexpr int N_PLANETS = 10;
constexpr int N_MASSES = 15;

// ------------------------------------------------------------------------------------------
// host copy of the loaded SPK segments (type 2 only), in load order
// ------------------------------------------------------------------------------------------
struct HostSeg {
    int64_t obj_id, center_id;
    int frame_code;
    int type;                 // 2, 3 (Chebyshev) or 1, 21 (modified difference arrays)
    double jd_start, jd_end;  // JD
    double start_s;           // jd_to_spice_jd(jd_start)
    double intlen;            // types 2, 3
    int64_t n_coef, rsize, n_rec;  // types 1, 21: n_coef = MAXDIM, rsize = 4 MAXDIM + 11
    std::vector<double> data;  // the DAF array
};

// Every record of a type 1 / 21 segment must keep the interpolation inside its arrays: the
// device kernels index by these orders without further checks (SPKE21 reads the same).
static bool mda_records_valid(const HostSeg& seg) {
    const int64_t md = seg.n_coef, rl = seg.rsize;
    const double* ep = seg.data.data() + seg.n_rec * rl;
    for (int64_t r = 0; r < seg.n_rec; ++r) {
        const double* rec = seg.data.data() + r * rl;
        for (int64_t q = 0; q < rl; ++q)
            if (!std::isfinite(rec[q])) return false;
        const double kqm = rec[4 * md + 7];
        if (kqm != std::floor(kqm) || kqm < 2.0 || kqm > (double)std::min<int64_t>(md + 1, 26)) return false;
        const int64_t kqmax1 = (int64_t)kqm;
        for (int c = 0; c < 3; ++c) {
            const double kq = rec[4 * md + 8 + c];
            if (kq != std::floor(kq) || kq < 0.0 || kq > (double)(kqmax1 - 1)) return false;
        }
        for (int64_t j = 0; j < kqmax1 - 2; ++j)
            if (rec[1 + j] == 0.0) return false;
        if (!std::isfinite(ep[r]) || (r > 0 && ep[r] < ep[r - 1])) return false;
    }
    return true;
}

struct DevState {
    int version = -1;       // ephemeris version resident on this device
    bool tables = false;
    double* facets = nullptr;  // thermal-model shape: 2048 unit normals, cos/sin latitude, 5 x 2048
    double* pool = nullptr;
    size_t pool_cap = 0;
    // grow-only staging buffers for host-pointer calls
    std::vector<std::pair<void*, size_t>> bufs;
};

static std::mutex g_mu;
static bool g_device_ready = false;  // kete_b200_init has run: loads upload eagerly
static LaunchConfig g_launch;
LaunchConfig& launch_config() { return g_launch; }
static std::vector<HostSeg> g_segs;
static int g_version = 0;
static int g_skipped = 0;
static std::map<int, DevState> g_dev;
static EphemConst g_eph;  // host image of the constant table (pool pointer set per device)
static std::vector<double> g_pool_host;
static std::map<int64_t, int> g_slot_of;  // naif id -> slot

static double spice_jds_to_jd(double s) { return s / 86400.0 + 2451545.0; }
static double jd_to_spice_jd(double jd) { return (jd - 2451545.0) * 86400.0; }

static int32_t rd_i32(const uint8_t* p, bool le) {
    uint32_t v;
    if (le)
        v = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    else
        v = (uint32_t)p[3] | ((uint32_t)p[2] << 8) | ((uint32_t)p[1] << 16) | ((uint32_t)p[0] << 24);
    return (int32_t)v;
}
static double rd_f64(const uint8_t* p, bool le) {
    uint8_t b[8];
    for (int i = 0; i < 8; ++i) b[i] = le ? p[i] : p[7 - i];
    double d;
    std::memcpy(&d, b, 8);
    return d;
}

static int parse_daf(const uint8_t* buf, int64_t n, std::vector<HostSeg>& out, int& skipped) {
    if (n < 1024) return set_error(KETE_B200_E_IO, "DAF file shorter than one record");
    if (std::strncmp((const char*)buf, "DAF/", 4) != 0 && std::strncmp((const char*)buf, "NAIF", 4) != 0)
        return set_error(KETE_B200_E_IO, "not a DAF file");
    char kind[4] = {0};
    for (int i = 0; i < 3; ++i) kind[i] = (char)toupper(buf[4 + i]);
    if (std::strncmp(kind, "SPK", 3) != 0) return set_error(KETE_B200_E_IO, "DAF file is not an SPK");
    bool le;
    if (std::strncmp((const char*)buf + 88, "LTL-IEEE", 8) == 0)
        le = true;
    else if (std::strncmp((const char*)buf + 88, "BIG-IEEE", 8) == 0)
        le = false;
    else
        return set_error(KETE_B200_E_IO, "Expected little or big endian in DAF file, found neither");
    const int nd = rd_i32(buf + 8, le), ni = rd_i32(buf + 12, le);
    if (nd != 2 || ni != 6) return set_error(KETE_B200_E_IO, "SPK File incorrectly Formatted.");
    const int summary_size = nd + (ni + 1) / 2;
    int next = rd_i32(buf + 76, le);
    int guard = 0;
    while (next != 0) {
        if (++guard > 100000) return set_error(KETE_B200_E_IO, "DAF summary chain does not end");
        const int64_t off = 1024LL * (next - 1);
        if (off < 0 || off + 1024 > n) return set_error(KETE_B200_E_IO, "DAF summary record outside the file");
        const uint8_t* rec = buf + off;
        next = (int)rd_f64(rec, le);
        const int n_sum = (int)rd_f64(rec + 16, le);
        if (n_sum < 0 || 24 + (int64_t)n_sum * summary_size * 8 > 1024)
            return set_error(KETE_B200_E_IO, "DAF summary record corrupt");
        for (int k = 0; k < n_sum; ++k) {
            const uint8_t* s = rec + 24 + (int64_t)k * summary_size * 8;
            const double f0 = rd_f64(s, le), f1 = rd_f64(s + 8, le);
            int32_t iv[6];
            for (int q = 0; q < 6; ++q) iv[q] = rd_i32(s + 16 + 4 * q, le);
            const int64_t a0 = iv[4], a1 = iv[5];
            const int64_t nf = a1 - a0 + 1;
            if (a0 < 1 || nf <= 4 || 8 * (a0 - 1) + 8 * nf > n)
                return set_error(KETE_B200_E_IO, "SPK array outside the file");
            const int type = iv[3];
            if (type != 2 && type != 3 && type != 1 && type != 21) {
                ++skipped;
                continue;
            }
            HostSeg seg;
            seg.obj_id = iv[0];
            seg.center_id = iv[1];
            seg.frame_code = iv[2];
            seg.type = type;
            seg.jd_start = spice_jds_to_jd(f0);
            seg.jd_end = spice_jds_to_jd(f1);
            seg.start_s = jd_to_spice_jd(seg.jd_start);
            seg.data.resize((size_t)nf);
            for (int64_t q = 0; q < nf; ++q) seg.data[q] = rd_f64(buf + 8 * (a0 - 1) + 8 * q, le);
            if (type == 2 || type == 3) {
                // From<DafArray> for SpkSegmentType2 / 3 (spk_segments.rs:379-397, 482-498)
                const int per = type == 2 ? 3 : 6;
                seg.rsize = (int64_t)seg.data[nf - 2];
                seg.intlen = seg.data[nf - 3];
                seg.n_coef = (seg.rsize - 2) / per;
                if (seg.rsize < 2 + 2 * per || per * seg.n_coef + 2 != seg.rsize)
                    return set_error(KETE_B200_E_IO,
                                     "File incorrectly formatted, found number of Chebyshev "
                                     "coefficients doesn't match expected");
                seg.n_rec = (nf - 4) / seg.rsize;
                if (seg.n_rec < 1 || !(seg.intlen > 0.0))
                    return set_error(KETE_B200_E_IO, "Chebyshev segment without records");
            } else {
                // From<DafArray> for SpkSegmentType1 / 21 (spk_segments.rs:302-308, 971-984)
                const double nr = seg.data[nf - 1];
                const double md = type == 1 ? 15.0 : seg.data[nf - 2];
                if (!(nr >= 1.0 && nr < 1e9) || !(md >= 1.0 && md <= 25.0) || md != std::floor(md))
                    return set_error(KETE_B200_E_IO, "SPK File contains segments of type " +
                                                         std::to_string(type) +
                                                         " has invalid contents.");
                seg.n_rec = (int64_t)nr;
                seg.n_coef = (int64_t)md;
                seg.rsize = 4 * seg.n_coef + 11;
                seg.intlen = 0.0;
                if (seg.n_rec * (seg.rsize + 1) > nf || !mda_records_valid(seg))
                    return set_error(KETE_B200_E_IO, "SPK File contains segments of type " +
                                                         std::to_string(type) +
                                                         " has invalid contents.");
            }
            out.push_back(std::move(seg));
        }
    }
    return 0;
}

// Fast-path plan for the first n_force entries of the force table: the evaluation order
// (a centre is evaluated before the bodies chained through it, again whenever it changes),
// each item's first segment, and the time window where all those segments cover and share
// FAST_NC coefficients.
static void build_fast_plan(int n_force, FastPlan& P) {
    std::memset(&P, 0, sizeof P);
    if (n_force <= 0) return;
    int n = 0;
    double lo = -1e300, hi = 1e300;
    bool ok = true;
    auto add = [&](int slot, int role) {
        if (n >= MAX_ITEMS || g_eph.slot[slot].count < 1) {
            ok = false;
            return;
        }
        const int seg = g_eph.slot[slot].first;
        const SegDesc& d = g_eph.seg[seg];
        if (d.type != 2 || d.n_pad != FAST_NC) ok = false;
        lo = std::max(lo, d.jd_start);
        hi = std::min(hi, d.jd_end);
        FastItem& I = P.item[n];
        I.offset = d.offset;
        I.start_s = d.start_s;
        I.inv_intlen = d.inv_intlen;
        I.n_rec = (double)d.n_rec;
        I.rsize = d.rsize;
        I.role = role;
        if (role >= 0) {
            const ForceEntry& fe = g_eph.force[role];
            I.mass = fe.mass;
            I.radius = fe.radius;
            I.kind = fe.kind;
            I.naif_id = fe.naif_id;
            I.chained = g_eph.slot[slot].parent_slot >= 0 ? 1 : 0;
        }
        ++n;
    };
    auto needs_velocity = [&](int b) {
        const int k = g_eph.force[b].kind;
        return k == FK_SUN || k == FK_JUPITER;
    };
    // bodies whose velocity enters the force, evaluated first (two at a time)
    for (int b = 0; b < n_force && ok; ++b) {
        if (!needs_velocity(b)) continue;
        if (g_eph.slot[g_eph.force[b].slot].parent_slot >= 0) ok = false;  // kept simple
        add(g_eph.force[b].slot, b);
    }
    P.n_vel = n;
    P.sun_vel = -1;
    for (int it = 0; it < n; ++it)
        if (P.item[it].kind == FK_SUN) P.sun_vel = it;
    // the others in the reference's order, each centre before the first body chained to it
    int current_parent = -1;
    for (int b = 0; b < n_force && ok; ++b) {
        if (needs_velocity(b)) continue;
        const int slot = g_eph.force[b].slot;
        const int parent = g_eph.slot[slot].parent_slot;
        if (parent >= 0 && parent != current_parent) {
            add(parent, -1);
            current_parent = parent;
        }
        add(slot, b);
    }
    while (ok && n > P.n_vel && (n - P.n_vel) % 3 != 0) add(g_eph.force[0].slot, -2);
    P.n_items = n;
    P.lo = lo;
    P.hi = hi;
    P.ok = (ok && n > 0 && lo <= hi) ? 1 : 0;
}

// Build the slot / segment / force tables and the device record pool from g_segs.
static int rebuild_tables() {
    std::memset(&g_eph, 0, sizeof g_eph);
    g_pool_host.clear();
    g_slot_of.clear();
    // slots in order of first appearance; segments grouped per body, load order kept
    std::vector<int64_t> ids;
    for (const auto& s : g_segs)
        if (!g_slot_of.count(s.obj_id)) {
            g_slot_of[s.obj_id] = (int)ids.size();
            ids.push_back(s.obj_id);
        }
    if ((int)ids.size() > MAX_SLOT) return set_error(KETE_B200_E_UNSUPPORTED, "too many SPK bodies for the device table");
    if ((int)g_segs.size() > MAX_SEG) return set_error(KETE_B200_E_UNSUPPORTED, "too many SPK segments for the device table");
    // coefficient blocks padded to one common width when every segment fits the fast path's
    // FAST_NC, so mixed coefficient counts (as in DE440s) still take it: the extra zero
    // coefficients add exactly nothing to the sums
    int64_t max_coef = 0;
    for (const auto& sg : g_segs)
        if (sg.type == 2) max_coef = std::max<int64_t>(max_coef, sg.n_coef);
    const bool common_pad = max_coef <= FAST_NC;
    int nseg = 0;
    for (size_t si = 0; si < ids.size(); ++si) {
        Slot& sl = g_eph.slot[si];
        sl.naif_id = (int32_t)ids[si];
        sl.first = nseg;
        sl.count = 0;
        sl.center_id = -1;
        for (const auto& s : g_segs) {
            if (s.obj_id != ids[si]) continue;
            if (s.frame_code != 1)
                return set_error(KETE_B200_E_UNSUPPORTED,
                                 "SPK segment for body " + std::to_string(s.obj_id) +
                                     " is not in the J2000 equatorial frame (code 1)");
            if (sl.count == 0) sl.center_id = (int32_t)s.center_id;
            else if (sl.center_id != s.center_id)
                return set_error(KETE_B200_E_UNSUPPORTED, "body with segments about different centres");
            SegDesc& d = g_eph.seg[nseg];
            d.jd_start = s.jd_start;
            d.jd_end = s.jd_end;
            d.start_s = s.start_s;
            d.intlen = s.intlen;
            d.inv_intlen = s.intlen > 0.0 ? 1.0 / s.intlen : 0.0;
            d.n_coef = (int32_t)s.n_coef;
            d.n_rec = (int32_t)s.n_rec;
            d.type = s.type;
            d.offset = (int64_t)g_pool_host.size();
            d.epoch_offset = 0;
            if (s.type == 1 || s.type == 21) {
                // records as stored, then the final epochs
                d.n_pad = 0;
                d.rsize = (int32_t)s.rsize;
                g_pool_host.insert(g_pool_host.end(), s.data.begin(),
                                   s.data.begin() + s.n_rec * (s.rsize + 1));
                d.epoch_offset = d.offset + s.n_rec * s.rsize;
                ++sl.count;
                ++nseg;
                continue;
            }
            if (s.type == 3) {
                d.n_pad = (int32_t)((s.n_coef + 1) & ~1LL);
                d.rsize = 4 + 6 * d.n_pad;
                for (int64_t r = 0; r < s.n_rec; ++r) {
                    const double* rec = s.data.data() + r * s.rsize;
                    const double mid = rec[0], rad = rec[1];
                    g_pool_host.push_back(mid);
                    g_pool_host.push_back(rad);
                    g_pool_host.push_back(1.0 / rad);
                    g_pool_host.push_back(86400.0 / AU_KM);  // spk_segments.rs:472
                    for (int c = 0; c < 6; ++c) {
                        for (int64_t q = 0; q < s.n_coef; ++q) g_pool_host.push_back(rec[2 + c * s.n_coef + q]);
                        for (int64_t q = s.n_coef; q < d.n_pad; ++q) g_pool_host.push_back(0.0);
                    }
                }
                ++sl.count;
                ++nseg;
                continue;
            }
            d.n_pad = common_pad ? FAST_NC : (int32_t)((s.n_coef + 1) & ~1LL);
            d.rsize = 4 + 3 * d.n_pad;
            for (int64_t r = 0; r < s.n_rec; ++r) {
                const double* rec = s.data.data() + r * s.rsize;
                const double mid = rec[0], rad = rec[1];
                g_pool_host.push_back(mid);
                g_pool_host.push_back(rad);
                g_pool_host.push_back(1.0 / rad);
                g_pool_host.push_back(86400.0 / rad / AU_KM);  // spk_segments.rs:366
                for (int c = 0; c < 3; ++c) {
                    for (int64_t q = 0; q < s.n_coef; ++q) g_pool_host.push_back(rec[2 + c * s.n_coef + q]);
                    for (int64_t q = s.n_coef; q < d.n_pad; ++q) g_pool_host.push_back(0.0);
                }
            }
            ++sl.count;
            ++nseg;
        }
    }
    for (size_t si = 0; si < ids.size(); ++si) {
        Slot& sl = g_eph.slot[si];
        sl.parent_slot = -1;
        if (sl.center_id != 0) {
            auto it = g_slot_of.find(sl.center_id);
            sl.parent_slot = it == g_slot_of.end() ? -2 : it->second;  // -2: centre not loaded
        }
    }
    g_eph.n_seg = nseg;
    g_eph.n_slot = (int32_t)ids.size();
    // force plan (PLANETS / MASSES).  A body is usable when its chain reaches the
    // barycentre within one intermediate centre.
    auto usable = [&](int64_t id) -> int {
        auto it = g_slot_of.find(id);
        if (it == g_slot_of.end()) return -1;
        const Slot& sl = g_eph.slot[it->second];
        if (sl.parent_slot == -1) return it->second;
        if (sl.parent_slot < 0) return -1;
        if (g_eph.slot[sl.parent_slot].parent_slot != -1) return -1;
        return it->second;
    };
    int nf = 0;
    bool planets_ok = true, all_ok = true;
    for (int b = 0; b < N_MASSES; ++b) {
        const int slot = usable(MASSES[b].id);
        if (slot < 0) {
            if (b < N_PLANETS) planets_ok = false;
            all_ok = false;
            continue;
        }
        if (!all_ok && b >= N_PLANETS) continue;
        ForceEntry& f = g_eph.force[nf++];
        f.mass = MASSES[b].mass_ratio == 1.0 ? GMS : MASSES[b].mass_ratio * GMS;
        f.radius = MASSES[b].radius;
        f.slot = slot;
        f.kind = MASSES[b].kind;
        f.naif_id = (int32_t)MASSES[b].id;
    }
    g_eph.n_force_planets = planets_ok ? N_PLANETS : 0;
    g_eph.n_force_all = (planets_ok && all_ok) ? N_MASSES : 0;
    build_fast_plan(g_eph.n_force_planets, g_eph.fast_planets);
    build_fast_plan(g_eph.n_force_all, g_eph.fast_all);
    g_eph.sun_slot = g_slot_of.count(10) ? g_slot_of[10] : -1;
    g_eph.loaded = 1;
    ++g_version;
    return 0;
}

static int ensure_tables(DevState& ds) {
    if (ds.tables) return 0;
    Tables t;
    std::memset(&t, 0, sizeof t);
    t.rot_c = std::cos(0.40909280422232897);
    t.rot_s = std::sin(0.40909280422232897);
    const double sp[8] = {0.0, 0.05626256053692215, 0.18024069173689236, 0.3526247171131696,
                          0.5471536263305554, 0.7342101772154105, 0.8853209468390958,
                          0.9775206135612875};
    for (int i = 0; i < 8; ++i) t.spacing[i] = sp[i];
    for (int i = 0; i < 7; ++i) {
        t.w[i] = 1.0 / (double)((i + 2) * (i + 3));
        t.u[i] = 1.0 / (double)(i + 2);
    }
    for (int i = 0; i < 7; ++i)
        for (int j = 0; j < 7; ++j) t.c[i][j] = i == j ? 1.0 : 0.0;
    for (int idx = 0; idx < 7; ++idx) {
        if (idx > 0) t.c[idx][0] = -sp[idx] * t.c[idx - 1][0];
        for (int idy = 1; idy < idx; ++idy)
            t.c[idx][idy] = t.c[idx - 1][idy - 1] - sp[idx] * t.c[idx - 1][idy];
    }
    auto powi_h = [](double x, int n) {  // LLVM powi expansion, as on the device
        double res = 1.0, sq = x;
        bool have = false;
        for (int v = n; v; v >>= 1) {
            if (v & 1) {
                res = have ? res * sq : sq;
                have = true;
            }
            if (v >> 1) sq = sq * sq;
        }
        return res;
    };
    for (int j = 1; j < 8; ++j) {
        for (int k = 0; k < 7; ++k) {
            t.w_pow[j][k] = powi_h(sp[j], 1 + k) * t.w[k];
            t.u_pow[j][k] = powi_h(sp[j], 1 + k) * t.u[k];
        }
        t.frac2[j] = powi_h(sp[j], 2);
        t.inv_frac[j] = 1.0 / sp[j];
        for (int z = 1; z < j; ++z) t.inv_diff[j][z] = 1.0 / (sp[j] - sp[z]);
    }
    // the corrector's map from node evaluations to b, b = P (E - a), column by column
    for (int col = 0; col < 7; ++col) {
        double g[7];
        for (int j = 1; j < 8; ++j) {
            double gk = (j - 1 == col ? 1.0 : 0.0) * t.inv_frac[j];
            for (int z = 1; z < j; ++z) gk = (gk - g[z - 1]) * t.inv_diff[j][z];
            g[j - 1] = gk;
        }
        for (int jj = 0; jj < 7; ++jj) {
            double s2 = g[jj];
            for (int k = jj + 1; k < 7; ++k) s2 += t.c[k][jj] * g[k];
            t.adj_p[jj][col] = s2;
        }
    }
    // SIMPLE_PLANETS: MASSES 0, 1, 2, the Earth-Moon barycentre (EM_BARY,
    // gravity.rs:137-142), MASSES 5-9
    {
        const int from_masses[9] = {0, 1, 2, -1, 5, 6, 7, 8, 9};
        for (int k = 0; k < 9; ++k) {
            if (from_masses[k] >= 0) {
                const GravEntry& e = MASSES[from_masses[k]];
                t.simple_mass[k] = e.mass_ratio == 1.0 ? GMS : e.mass_ratio * GMS;
                t.simple_radius[k] = e.radius;
                t.simple_kind[k] = e.kind;
                t.simple_naif[k] = (int32_t)e.id;
            } else {
                t.simple_mass[k] = (3.00348961546514e-06 + 3.69430335010988e-08) * GMS;
                t.simple_radius[k] = 385000.0 / AU_KM;
                t.simple_kind[k] = FK_PLAIN;
                t.simple_naif[k] = 3;
            }
        }
    }
    // a(tau) = a0 + sum_k b_k tau^(k+1) over the previous step, re-expanded about its end
    // with the new step's scale q: b'_m = q^(m+1) sum_{k>=m} C(k+1, m+1) b_k
    for (int m = 0; m < 7; ++m)
        for (int k = 0; k < 7; ++k) {
            double cnk = 0.0;
            if (k >= m) {
                cnk = 1.0;
                for (int i = 0; i < m + 1; ++i) cnk = cnk * (double)(k + 1 - i) / (double)(i + 1);
            }
            t.shift_c[m][k] = cnk;
        }
    int rc = upload_tables(t);
    if (rc) return rc;
    // DEFAULT_SHAPE: 2048-facet Fibonacci lattice, total area 1 (flux/shapes.rs:9, 42-66)
    {
        const double TAUD = 6.283185307179586, GOLDEN_RATIO = 1.618033988749894, EPS = 0.36;
        const double nf = (double)N_FACETS;
        std::vector<double> f(5 * N_FACETS);
        for (int idx = 0; idx < N_FACETS; ++idx) {
            const double theta = TAUD * (double)idx / GOLDEN_RATIO;
            const double phi = std::acos(1.0 - 2.0 * ((double)idx + EPS) / (nf - 1.0 + 2.0 * EPS));
            f[idx] = std::cos(theta) * std::sin(phi);
            f[N_FACETS + idx] = std::sin(theta) * std::sin(phi);
            f[2 * N_FACETS + idx] = std::cos(phi);
            // cos and sin of the facet latitude for the FRM: the host's asin, as frm.rs:26
            // evaluates it
            const double lat = std::asin(f[2 * N_FACETS + idx]);
            f[3 * N_FACETS + idx] = std::cos(lat);
            f[4 * N_FACETS + idx] = std::sin(lat);
        }
        if ((rc = cuda_check(counted_malloc((void**)&ds.facets, f.size() * sizeof(double)), "cudaMalloc facets")))
            return rc;
        if ((rc = cuda_check(cudaMemcpy(ds.facets, f.data(), f.size() * sizeof(double),
                                        cudaMemcpyHostToDevice),
                             "upload facets")))
            return rc;
    }
    ds.tables = true;
    return 0;
}

static int current_device(int& dev) { return cuda_check(cudaGetDevice(&dev), "cudaGetDevice"); }

// Make the latest ephemeris resident on the current device.
static int ensure_device(DevState*& out) {
    int dev;
    int rc = current_device(dev);
    if (rc) return rc;
    DevState& ds = g_dev[dev];
    if ((rc = ensure_tables(ds))) return rc;
    if (ds.version != g_version) {
        const size_t bytes = g_pool_host.size() * sizeof(double);
        if (bytes > ds.pool_cap) {
            if (ds.pool) cudaFree(ds.pool);
            ds.pool = nullptr;
            ds.pool_cap = 0;
            if ((rc = cuda_check(counted_malloc((void**)&ds.pool, bytes), "cudaMalloc ephemeris pool"))) return rc;
            ds.pool_cap = bytes;
        }
        if (bytes && (rc = cuda_check(cudaMemcpy(ds.pool, g_pool_host.data(), bytes, cudaMemcpyHostToDevice),
                                      "upload ephemeris pool")))
            return rc;
        EphemConst e = g_eph;
        e.pool = ds.pool;
        if ((rc = upload_ephem(e))) return rc;
        ds.version = g_version;
    }
    out = &ds;
    return 0;
}

// grow-only staging buffer `k` of at least `bytes`
static int staging(DevState& ds, size_t k, size_t bytes, void** p) {
    if (ds.bufs.size() <= k) ds.bufs.resize(k + 1, {nullptr, 0});
    auto& b = ds.bufs[k];
    if (b.second < bytes) {
        if (b.first) cudaFree(b.first);
        b.first = nullptr;
        b.second = 0;
        const size_t want = bytes < 256 ? 256 : bytes;
        int rc = cuda_check(counted_malloc((void**)&b.first, want), "cudaMalloc staging buffer");
        if (rc) return rc;
        b.second = want;
    }
    *p = b.first;
    return 0;
}

// chain of slots from `center` up to the barycentre (empty for centre 0)
static int center_chain(int64_t center, CenterChain& ch) {
    ch.len = 0;
    int64_t c = center;
    while (c != 0) {
        auto it = g_slot_of.find(c);
        if (it == g_slot_of.end() || ch.len >= 3)
            return set_error(KETE_B200_E_NO_EPHEMERIS,
                             "SPK files are missing information to be able to map from obj " +
                                 std::to_string(center) + " to obj 0");
        ch.slot[ch.len++] = it->second;
        c = g_eph.slot[it->second].center_id;
    }
    return 0;
}

static int check_frame(int frame) {
    if (frame != FRAME_EQUATORIAL && frame != FRAME_ECLIPTIC)
        return set_error(KETE_B200_E_UNSUPPORTED, "frame must be equatorial (1) or ecliptic (2)");
    return 0;
}

// Host-pointer staging helper: copy in, run, copy out.
struct Stager {
    DevState& ds;
    cudaStream_t st;
    int on_device;
    size_t slot = 0;
    int rc = 0;
    std::vector<std::tuple<void*, const void*, size_t>> outs;  // host dst, dev src, bytes
    template <class T>
    T* in(const T* host, size_t count) {
        if (!host || rc) return const_cast<T*>(host);
        if (on_device) return const_cast<T*>(host);
        void* d;
        if ((rc = staging(ds, slot++, count * sizeof(T), &d))) return nullptr;
        rc = cuda_check(cudaMemcpyAsync(d, host, count * sizeof(T), cudaMemcpyHostToDevice, st), "copy inputs to device");
        return (T*)d;
    }
    template <class T>
    T* out(T* host, size_t count) {
        if (!host || rc) return host;
        if (on_device) return host;
        void* d;
        if ((rc = staging(ds, slot++, count * sizeof(T), &d))) return nullptr;
        outs.emplace_back((void*)host, d, count * sizeof(T));
        return (T*)d;
    }
    int finish() {
        if (rc) return rc;
        for (auto& o : outs)
            if ((rc = cuda_check(cudaMemcpyAsync(std::get<0>(o), std::get<1>(o), std::get<2>(o),
                                                 cudaMemcpyDeviceToHost, st),
                                 "copy results to host")))
                return rc;
        if (!on_device) rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize");
        return rc;
    }
};

// The node-kernel variant to launch for a force list: the cached variants (6-8 warp-
// synchronous, 9-10 warp-pooled) only pay off with the body-position cache, so a plan that
// does not fit it (or no fast plan) runs the uncached step-end twins (3-5), which integrate
// identically.
int nodes_variant_for(int variant, int n_force) {
    if (variant < 6) return variant;
    const FastPlan& P = n_force == g_eph.n_force_planets ? g_eph.fast_planets : g_eph.fast_all;
    if (variant >= 9)  // pooled: the uncached step-end form of the same register budget
        return (!P.ok || pool_plan_doubles(P) > POOL_CACHE_DOUBLES) ? variant - 5 : variant;
    if (!P.ok || fast_plan_cache_doubles(P) > EPH_CACHE) return variant - 3;
    return variant;
}

// The window a variant needs its objects' spans inside (the warp-pooled kernels: the fast
// plan's), or [-inf, inf].
void nodes_window(int variant, int n_force, double& lo, double& hi) {
    const FastPlan& P = n_force == g_eph.n_force_planets ? g_eph.fast_planets : g_eph.fast_all;
    lo = -INFINITY;
    hi = INFINITY;
    if (variant >= 9) {
        lo = P.lo;
        hi = P.hi;
    }
}

// Everything the allocation-free entry point needs, read under the lock without allocating:
// the ephemeris must already be resident on the current device.
int noalloc_snapshot(int include_asteroids, int64_t center, NBodyArgs& a, LaunchConfig& cfg,
                     NodesPlan& plan) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    int dev = 0;
    int rc = current_device(dev);
    if (rc) return rc;
    auto it = g_dev.find(dev);
    if (it == g_dev.end() || !it->second.tables || it->second.version != g_version)
        return set_error(KETE_B200_E_NO_EPHEMERIS,
                         "the loaded SPK is not resident on this device yet: call kete_b200_init "
                         "on it before loading, or make one allocating call first");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0)
        return set_error(KETE_B200_E_NO_EPHEMERIS, "loaded SPKs lack a perturbing body");
    if ((rc = center_chain(center, a.chain))) return rc;
    a.n_force = n_force;
    cfg = g_launch;
    cfg.nodes_variant = nodes_variant_for(cfg.nodes_variant, n_force);
    plan.general_variant = nodes_variant_for(7, n_force);
    nodes_window(cfg.nodes_variant, n_force, plan.lo, plan.hi);
    return 0;
}

}  // namespace kb

using namespace kb;

extern "C" {

int kete_b200_version(void) { return 100; }

int64_t kete_b200_kernel_launches(void) { return g_kernel_launches.load(); }

const char* kete_b200_last_error(void) { return g_last_error.c_str(); }

int kete_b200_init(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = cuda_check(cudaSetDevice(device), "cudaSetDevice");
    if (rc) return rc;
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    // load the kernels and resolve the fixed scratch of the allocation-free entry point now,
    // so that its calls on this device load no module (which could allocate) themselves
    if ((rc = preload_nodes_kernels())) return rc;
    if ((rc = preload_order_kernels())) return rc;
    if ((rc = noalloc_prepare())) return rc;
    g_device_ready = true;
    return 0;
}

int64_t kete_b200_device_allocations(void) { return g_device_allocations.load(); }

int kete_b200_spk_load_buffer(const uint8_t* bytes, int64_t n_bytes) {
    if (!bytes || n_bytes <= 0) return set_error(KETE_B200_E_ARGUMENT, "empty SPK buffer");
    std::lock_guard<std::mutex> lk(g_mu);
    std::vector<HostSeg> segs;
    int skipped = 0;
    int rc = parse_daf(bytes, n_bytes, segs, skipped);
    if (rc) return rc;
    for (auto& s : segs) g_segs.push_back(std::move(s));
    g_skipped += skipped;
    if ((rc = rebuild_tables())) return rc;
    if (g_device_ready) {  // make the new ephemeris resident on the current device now
        DevState* ds;
        if ((rc = ensure_device(ds))) return rc;
    }
    return 0;
}

int kete_b200_spk_load_file(const char* path) {
    if (!path) return set_error(KETE_B200_E_ARGUMENT, "null path");
    std::ifstream f(path, std::ios::binary);
    if (!f) return set_error(KETE_B200_E_IO, std::string("cannot open ") + path);
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    return kete_b200_spk_load_buffer(buf.data(), (int64_t)buf.size());
}

int kete_b200_spk_reset(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_segs.clear();
    g_skipped = 0;
    g_slot_of.clear();
    std::memset(&g_eph, 0, sizeof g_eph);
    g_pool_host.clear();
    ++g_version;
    return 0;
}

int kete_b200_spk_skipped(void) { return g_skipped; }

int kete_b200_spk_loaded_ids(int64_t* ids, int max) {
    std::lock_guard<std::mutex> lk(g_mu);
    int k = 0;
    for (int s = 0; s < g_eph.n_slot; ++s) {
        if (ids && k < max) ids[k] = g_eph.slot[s].naif_id;
        ++k;
    }
    return k;
}

int kete_b200_spk_get_states(int64_t n, int64_t id, const double* jd, int64_t center, int frame,
                             double* out6, int32_t* status, int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!jd || !out6 || !status))) return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = check_frame(frame);
    if (rc) return rc;
    auto it = g_slot_of.find(id);
    if (it == g_slot_of.end())
        return set_error(KETE_B200_E_NO_EPHEMERIS,
                         "Object (" + std::to_string(id) + ") does not have an SPK record");
    CenterChain ch;
    if ((rc = center_chain(center, ch))) return rc;
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_jd = S.in(jd, (size_t)n);
    double* d_out = S.out(out6, (size_t)n * 6);
    int32_t* d_st = S.out(status, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_spk_states(n, it->second, d_jd, ch, frame, d_out, d_st, st))) return rc;
    return S.finish();
}

int kete_b200_propagate_two_body(int64_t n, const double* pos, const double* vel,
                                 const double* jd0, const double* jd1, const double* observer_pos,
                                 double* out_pos, double* out_vel, double* out_jd, int32_t* status,
                                 int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!pos || !vel || !jd0 || !jd1 || !out_pos || !out_vel || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_pos = S.in(pos, 3 * (size_t)n);
    const double* d_vel = S.in(vel, 3 * (size_t)n);
    const double* d_jd0 = S.in(jd0, (size_t)n);
    const double* d_jd1 = S.in(jd1, (size_t)n);
    const double* d_obs = S.in(observer_pos, 3);
    double* d_op = S.out(out_pos, 3 * (size_t)n);
    double* d_ov = S.out(out_vel, 3 * (size_t)n);
    double* d_oj = S.out(out_jd, (size_t)n);
    int32_t* d_st = S.out(status, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_two_body(n, d_pos, d_vel, d_jd0, d_jd1, d_obs, d_op, d_ov, d_oj, d_st, st)))
        return rc;
    return S.finish();
}

int kete_b200_compute_stm(int64_t n, const double* pos, const double* vel, const double* jd0,
                          const double* jd1, double central_mass, const double* covariance,
                          double* out_pos, double* out_vel, double* out_stm, double* out_cov,
                          int32_t* status, int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!pos || !vel || !jd0 || !jd1 || !out_pos || !out_vel || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (!(central_mass > 0.0) || !std::isfinite(central_mass))
        return set_error(KETE_B200_E_ARGUMENT, "central_mass must be positive");
    if ((covariance == nullptr) != (out_cov == nullptr))
        return set_error(KETE_B200_E_ARGUMENT, "covariance and out_cov go together");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_pos = S.in(pos, 3 * (size_t)n);
    const double* d_vel = S.in(vel, 3 * (size_t)n);
    const double* d_jd0 = S.in(jd0, (size_t)n);
    const double* d_jd1 = S.in(jd1, (size_t)n);
    const double* d_cov = S.in(covariance, 36 * (size_t)n);
    double* d_op = S.out(out_pos, 3 * (size_t)n);
    double* d_ov = S.out(out_vel, 3 * (size_t)n);
    double* d_stm = S.out(out_stm, 36 * (size_t)n);
    double* d_oc = S.out(out_cov, 36 * (size_t)n);
    int32_t* d_st = S.out(status, (size_t)n);
    if (S.rc) return S.rc;
    // GM of the central body: kete's GMS for one solar mass (constants/gravity.rs:9)
    const double mu = central_mass == 1.0 ? GMS : GMS * central_mass;
    if ((rc = launch_two_body_stm(n, d_pos, d_vel, d_jd0, d_jd1, mu, d_cov, d_op, d_ov, d_stm, d_oc,
                                  d_st, st)))
        return rc;
    return S.finish();
}

int kete_b200_covariance_transform(int64_t n, int rows, int cols, const double* stm,
                                   const double* covariance, double* out_cov, int on_device,
                                   void* stream) {
    if (n < 0 || (n > 0 && (!stm || !covariance || !out_cov)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (rows < 1 || rows > 16 || cols < 1 || cols > 16)
        return set_error(KETE_B200_E_ARGUMENT, "rows and cols must be 1..16");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_stm = S.in(stm, (size_t)rows * cols * n);
    const double* d_cov = S.in(covariance, (size_t)cols * cols * n);
    double* d_out = S.out(out_cov, (size_t)rows * rows * n);
    if (S.rc) return S.rc;
    if ((rc = launch_covariance(n, rows, cols, d_stm, d_cov, d_out, st))) return rc;
    return S.finish();
}

int kete_b200_propagate_n_body(int64_t n, const double* pos, const double* vel, const double* jd0,
                               const double* jd1, int frame, int64_t center, int include_asteroids,
                               const double* nongrav, double* out_pos, double* out_vel,
                               int32_t* status, int32_t* impact_id, double* impact_jd,
                               double* min_dist, int32_t* counters, int mode, int on_device,
                               void* stream) {
    if (n < 0 || (n > 0 && (!pos || !vel || !jd0 || !jd1 || !out_pos || !out_vel || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = check_frame(frame);
    if (rc) return rc;
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0)
        return set_error(KETE_B200_E_NO_EPHEMERIS,
                         include_asteroids ? "loaded SPKs lack a perturbing asteroid or planet"
                                           : "loaded SPKs lack a planet, the Sun or the Moon");
    NBodyArgs a;
    std::memset(&a, 0, sizeof a);
    if ((rc = center_chain(center, a.chain))) return rc;
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    a.n = n;
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.jd0 = S.in(jd0, (size_t)n);
    a.jd1 = S.in(jd1, (size_t)n);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.frame = frame;
    a.n_force = n_force;
    a.out_pos = S.out(out_pos, 3 * (size_t)n);
    a.out_vel = S.out(out_vel, 3 * (size_t)n);
    a.status = S.out(status, (size_t)n);
    a.impact_id = S.out(impact_id, (size_t)n);
    a.impact_jd = S.out(impact_jd, (size_t)n);
    a.min_dist = S.out(min_dist, (size_t)n);
    a.counters = S.out(counters, 3 * (size_t)n);
    a.max_loops = g_launch.max_loops;
    if (S.rc) return S.rc;
    if (mode == KETE_B200_MODE_THREAD) {
        if ((rc = launch_nbody_thread(a, g_launch.thread_block, st))) return rc;
    } else if (mode == KETE_B200_MODE_NODES || mode == KETE_B200_MODE_AUTO) {
        // objects in order of their work (span in orbital periods), most first; scratch holds
        // the queue counter, the work histogram and the processing order
        void* q = nullptr;
        if ((rc = staging(*ds, 31, (ORDER_SCRATCH_HEADER + (size_t)n) * sizeof(int), &q)))
            return rc;
        const int variant = nodes_variant_for(g_launch.nodes_variant, a.n_force);
        double lo, hi;
        nodes_window(variant, a.n_force, lo, hi);
        if ((rc = launch_span_order(n, a.pos, a.vel, a.jd0, a.jd1, lo, hi,
                                    variant >= 9 ? a.nongrav : nullptr, (int*)q, st)))
            return rc;
        // refill: a persistent grid taking the next object from the queue
        if ((rc = launch_nodes_ordered(a, variant, nodes_variant_for(7, a.n_force),
                                       g_launch.nodes_refill != 0, (int*)q, st)))
            return rc;
    } else {
        return set_error(KETE_B200_E_ARGUMENT, "unknown propagation mode");
    }
    return S.finish();
}

int kete_b200_radau_central(int64_t n, const double* pos, const double* vel, const double* t0,
                            const double* t1, double* out_pos, double* out_vel, int32_t* status,
                            int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!pos || !vel || !t0 || !t1 || !out_pos || !out_vel || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_p = S.in(pos, 3 * (size_t)n);
    const double* d_v = S.in(vel, 3 * (size_t)n);
    const double* d_t0 = S.in(t0, (size_t)n);
    const double* d_t1 = S.in(t1, (size_t)n);
    double* d_op = S.out(out_pos, 3 * (size_t)n);
    double* d_ov = S.out(out_vel, 3 * (size_t)n);
    int32_t* d_st = S.out(status, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_radau_central(n, d_p, d_v, d_t0, d_t1, d_op, d_ov, d_st, st))) return rc;
    return S.finish();
}

int kete_b200_spk_accel(int64_t n, const double* jd, const double* pos, const double* vel,
                        int include_asteroids, const double* nongrav, int exact, double* out_acc,
                        int32_t* status, int32_t* impact_id, int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!jd || !pos || !vel || !out_acc || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0)
        return set_error(KETE_B200_E_NO_EPHEMERIS,
                         include_asteroids ? "loaded SPKs lack a perturbing asteroid or planet"
                                           : "loaded SPKs lack a planet, the Sun or the Moon");
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc || n == 0) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    AccelArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n;
    a.jd = S.in(jd, (size_t)n);
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.n_force = n_force;
    a.exact = exact ? 1 : 0;
    a.out = S.out(out_acc, 3 * (size_t)n);
    a.status = S.out(status, (size_t)n);
    a.impact_id = S.out(impact_id, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_accel(a, false, st))) return rc;
    return S.finish();
}

int kete_b200_vec_accel(int64_t n, int bodies, const double* massive, const double* pos,
                        const double* vel, const double* nongrav, int exact, double* out_acc,
                        int32_t* status, int32_t* impact_id, int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!massive || !pos || !vel || !out_acc || !status)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (bodies != KETE_B200_BODIES_PLANETS && bodies != KETE_B200_BODIES_MASSES &&
        bodies != KETE_B200_BODIES_SIMPLE_PLANETS)
        return set_error(KETE_B200_E_ARGUMENT, "unknown body list");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc || n == 0) return rc;
    AccelArgs a;
    std::memset(&a, 0, sizeof a);
    if (bodies == KETE_B200_BODIES_SIMPLE_PLANETS) {
        a.simple = 1;
        a.n_massive = 9;
    } else {
        a.n_massive = bodies == KETE_B200_BODIES_MASSES ? N_MASSES : N_PLANETS;
        for (int b = 0; b < a.n_massive; ++b) {
            ForceEntry& f = a.bodies[b];
            f.mass = MASSES[b].mass_ratio == 1.0 ? GMS : MASSES[b].mass_ratio * GMS;
            f.radius = MASSES[b].radius;
            f.slot = -1;
            f.kind = MASSES[b].kind;
            f.naif_id = (int32_t)MASSES[b].id;
        }
    }
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    a.n = n;
    a.massive = S.in(massive, 6 * (size_t)a.n_massive);
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.exact = exact ? 1 : 0;
    a.out = S.out(out_acc, 3 * (size_t)n);
    a.status = S.out(status, (size_t)n);
    a.impact_id = S.out(impact_id, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_accel(a, true, st))) return rc;
    return S.finish();
}

int kete_b200_hg_apparent_mag(int64_t n, const double* sun2obj, const double* sun2obs,
                              const double* h_mag, const double* g_param, double* out_mag,
                              int on_device, void* stream) {
    if (n < 0 || (n > 0 && (!sun2obj || !sun2obs || !h_mag || !g_param || !out_mag)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc || n == 0) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* a = S.in(sun2obj, 3 * (size_t)n);
    const double* b = S.in(sun2obs, 3 * (size_t)n);
    const double* h = S.in(h_mag, (size_t)n);
    const double* g = S.in(g_param, (size_t)n);
    double* o = S.out(out_mag, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_hg_mag(n, a, b, h, g, o, st))) return rc;
    return S.finish();
}

}  // extern "C"

namespace kb {

// NEATM (model 0) and FRM (model 1) share the facet sum; FRM ignores beaming.
static int thermal_model(int model, int64_t n, const double* sun2obj, const double* sun2obs,
                         const double* h_mag, const double* g_param, const double* diam,
                         const double* vis_albedo, const double* beaming,
                         const double* emissivity, int n_bands, const double* band_wavelength,
                         const double* band_albedos, const double* sun_correction,
                         const double* zero_mags, int wise_color_correction, double* fluxes,
                         double* thermal_fluxes, double* hg_fluxes, double* magnitudes,
                         double* v_mag, double* v_flux, int on_device, void* stream) {
    if (n_bands < 1 || n_bands > MAX_BANDS)
        return set_error(KETE_B200_E_ARGUMENT, "n_bands must be 1..8");
    if (!band_wavelength || !sun_correction) return set_error(KETE_B200_E_ARGUMENT, "null band table");
    if (wise_color_correction && n_bands != 4)
        return set_error(KETE_B200_E_ARGUMENT, "WISE colour correction needs the 4 WISE bands");
    if (n < 0 || (n > 0 && (!sun2obj || !sun2obs || !h_mag || !g_param || !diam || !vis_albedo ||
                            (model == 0 && !beaming) || !emissivity || !band_albedos || !fluxes ||
                            !thermal_fluxes || !hg_fluxes || !v_mag || !v_flux)))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc || n == 0) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    NeatmArgs a;
    std::memset(&a, 0, sizeof a);
    a.model = model;
    a.n = n;
    a.n_bands = n_bands;
    for (int b = 0; b < n_bands; ++b) {
        a.wavelength[b] = band_wavelength[b];
        a.sun_correction[b] = sun_correction[b];
        a.zero_mag[b] = zero_mags ? zero_mags[b] : 0.0;
        // black_body_flux's per-band constants (common.rs:139-154); bands below 10 nm
        // give no thermal flux
        const double wl_um = band_wavelength[b] * 1e-3;
        a.bb_k[b] = 1.43877688e4 / wl_um;
        a.bb_coef[b] = band_wavelength[b] < 10.0 ? 0.0 : 397.289171e17 / ((wl_um * wl_um) * wl_um);
    }
    a.have_zero_mags = zero_mags ? 1 : 0;
    a.wise_cc = wise_color_correction ? 1 : 0;
    a.facets = ds->facets;
    a.facet_area = 1.0 / (double)N_FACETS;
    Stager S{*ds, st, on_device};
    a.sun2obj = S.in(sun2obj, 3 * (size_t)n);
    a.sun2obs = S.in(sun2obs, 3 * (size_t)n);
    a.h_mag = S.in(h_mag, (size_t)n);
    a.g_param = S.in(g_param, (size_t)n);
    a.diam = S.in(diam, (size_t)n);
    a.vis_albedo = S.in(vis_albedo, (size_t)n);
    a.beaming = model == 0 ? S.in(beaming, (size_t)n) : nullptr;
    a.emissivity = S.in(emissivity, (size_t)n);
    a.band_albedo = S.in(band_albedos, (size_t)n_bands * n);
    a.fluxes = S.out(fluxes, (size_t)n_bands * n);
    a.thermal = S.out(thermal_fluxes, (size_t)n_bands * n);
    a.hg_fluxes = S.out(hg_fluxes, (size_t)n_bands * n);
    a.mags = S.out(magnitudes, (size_t)n_bands * n);
    a.v_mag = S.out(v_mag, (size_t)n);
    a.v_flux = S.out(v_flux, (size_t)n);
    if (S.rc) return S.rc;
    if ((rc = launch_neatm(a, st))) return rc;
    return S.finish();
}

}  // namespace kb

extern "C" {

int kete_b200_neatm(int64_t n, const double* sun2obj, const double* sun2obs, const double* h_mag,
                    const double* g_param, const double* diam, const double* vis_albedo,
                    const double* beaming, const double* emissivity, int n_bands,
                    const double* band_wavelength, const double* band_albedos,
                    const double* sun_correction, const double* zero_mags,
                    int wise_color_correction, double* fluxes, double* thermal_fluxes,
                    double* hg_fluxes, double* magnitudes, double* v_mag, double* v_flux,
                    int on_device, void* stream) {
    return kb::thermal_model(0, n, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, beaming,
                             emissivity, n_bands, band_wavelength, band_albedos, sun_correction,
                             zero_mags, wise_color_correction, fluxes, thermal_fluxes, hg_fluxes,
                             magnitudes, v_mag, v_flux, on_device, stream);
}

int kete_b200_frm(int64_t n, const double* sun2obj, const double* sun2obs, const double* h_mag,
                  const double* g_param, const double* diam, const double* vis_albedo,
                  const double* emissivity, int n_bands, const double* band_wavelength,
                  const double* band_albedos, const double* sun_correction,
                  const double* zero_mags, int wise_color_correction, double* fluxes,
                  double* thermal_fluxes, double* hg_fluxes, double* magnitudes, double* v_mag,
                  double* v_flux, int on_device, void* stream) {
    return kb::thermal_model(1, n, sun2obj, sun2obs, h_mag, g_param, diam, vis_albedo, nullptr,
                             emissivity, n_bands, band_wavelength, band_albedos, sun_correction,
                             zero_mags, wise_color_correction, fluxes, thermal_fluxes, hg_fluxes,
                             magnitudes, v_mag, v_flux, on_device, stream);
}

int kete_b200_propagate_n_body_stm(int64_t n, const double* pos, const double* vel,
                                   const double* jd0, int n_epochs, const double* epochs,
                                   int frame, int64_t center, int include_asteroids,
                                   const double* nongrav, double* out_state, double* out_stm,
                                   int32_t* status, int on_device, void* stream) {
    if (n < 0 || n_epochs < 1 || !epochs)
        return set_error(KETE_B200_E_ARGUMENT, "need n >= 0 and at least one epoch");
    if (n > 0 && (!pos || !vel || !jd0 || !out_state || !out_stm || !status))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = check_frame(frame);
    if (rc) return rc;
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0) return set_error(KETE_B200_E_NO_EPHEMERIS, "loaded SPKs lack a perturber");
    StmArgs a;
    std::memset(&a, 0, sizeof a);
    if ((rc = center_chain(center, a.chain))) return rc;
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    a.n = n;
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.jd0 = S.in(jd0, (size_t)n);
    a.n_epochs = n_epochs;
    a.epochs = S.in(epochs, (size_t)n_epochs);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.frame = frame;
    a.n_force = n_force;
    a.out_state = S.out(out_state, (size_t)n_epochs * 6 * n);
    a.out_stm = S.out(out_stm, (size_t)n_epochs * 48 * n);
    a.status = S.out(status, (size_t)n);
    a.max_loops = g_launch.max_loops;
    if (S.rc) return S.rc;
    if ((rc = launch_nbody_stm(a, g_launch.sens_form, st))) return rc;
    return S.finish();
}

static_assert(SENS_STRIDE == KETE_B200_CHECKPOINT_DOUBLES, "checkpoint size");
static_assert(FOV_STRIDE == KETE_B200_FOV_ROWS, "field table rows");
int kete_b200_checkpoint_doubles(void) { return KETE_B200_CHECKPOINT_DOUBLES; }

int kete_b200_propagate_n_body_checkpointed(int64_t n, const double* pos, const double* vel,
                                             const double* jd0, int n_epochs, const double* epochs,
                                             int frame, int64_t center, int include_asteroids,
                                             const double* nongrav, double* out_state,
                                             int32_t* status, int ckpt_capacity,
                                             double* checkpoints, int32_t* ckpt_count,
                                             int32_t* ckpt_segment, int on_device, void* stream) {
    if (n < 0 || n_epochs < 1 || !epochs || ckpt_capacity < 1)
        return set_error(KETE_B200_E_ARGUMENT, "need n >= 0, at least one epoch and a checkpoint capacity >= 1");
    if (n > 0 && (!pos || !vel || !jd0 || !out_state || !status || !checkpoints || !ckpt_count ||
                  !ckpt_segment))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = check_frame(frame);
    if (rc) return rc;
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0) return set_error(KETE_B200_E_NO_EPHEMERIS, "loaded SPKs lack a perturber");
    SensArgs a;
    std::memset(&a, 0, sizeof a);
    if ((rc = center_chain(center, a.chain))) return rc;
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    a.n = n;
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.jd0 = S.in(jd0, (size_t)n);
    a.n_epochs = n_epochs;
    a.epochs = S.in(epochs, (size_t)n_epochs);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.frame = frame;
    a.n_force = n_force;
    a.out_state = S.out(out_state, (size_t)n_epochs * 6 * n);
    a.status = S.out(status, (size_t)n);
    a.ckpt_cap = ckpt_capacity;
    a.ckpt = S.out(checkpoints, (size_t)n * ckpt_capacity * SENS_STRIDE);
    a.ckpt_count = S.out(ckpt_count, (size_t)n);
    a.ckpt_seg = S.out(ckpt_segment, (size_t)n_epochs * n);
    a.max_loops = g_launch.max_loops;
    if (S.rc) return S.rc;
    if ((rc = launch_sens_forward(a, st))) return rc;
    return S.finish();
}

int kete_b200_propagate_n_body_adjoint(int64_t n, int n_epochs, const double* epochs, int frame,
                                       int include_asteroids, const double* nongrav,
                                       int ckpt_capacity, const double* checkpoints,
                                       const int32_t* ckpt_count, const int32_t* ckpt_segment,
                                       const int32_t* status, const double* seed,
                                       double* out_grad, int32_t* grad_status, int on_device,
                                       void* stream) {
    if (n < 0 || n_epochs < 1 || !epochs || ckpt_capacity < 1)
        return set_error(KETE_B200_E_ARGUMENT, "need n >= 0, at least one epoch and a checkpoint capacity >= 1");
    if (n > 0 && (!checkpoints || !ckpt_count || !ckpt_segment || !status || !seed || !out_grad))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = check_frame(frame);
    if (rc) return rc;
    if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
    const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
    if (n_force == 0) return set_error(KETE_B200_E_NO_EPHEMERIS, "loaded SPKs lack a perturber");
    SensArgs a;
    std::memset(&a, 0, sizeof a);
    DevState* ds;
    if ((rc = ensure_device(ds))) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    a.n = n;
    a.n_epochs = n_epochs;
    a.epochs = S.in(epochs, (size_t)n_epochs);
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.frame = frame;
    a.n_force = n_force;
    a.ckpt_cap = ckpt_capacity;
    a.ckpt = const_cast<double*>(S.in(checkpoints, (size_t)n * ckpt_capacity * SENS_STRIDE));
    a.ckpt_count = const_cast<int32_t*>(S.in(ckpt_count, (size_t)n));
    a.ckpt_seg = const_cast<int32_t*>(S.in(ckpt_segment, (size_t)n_epochs * n));
    a.status = const_cast<int32_t*>(S.in(status, (size_t)n));
    a.seed = S.in(seed, (size_t)n_epochs * 6 * n);
    a.out_grad = S.out(out_grad, 8 * (size_t)n);
    a.grad_status = S.out(grad_status, (size_t)n);
    a.max_loops = g_launch.max_loops;
    if (S.rc) return S.rc;
    // per-object attempt records of the block being transposed (library scratch)
    void* rec;
    if ((rc = staging(*ds, 33, (size_t)n * (SENS_CK_ATTEMPTS + 1) * SENS_STRIDE * sizeof(double), &rec)))
        return rc;
    a.rec = (double*)rec;
    // the records of every checkpoint block, replayed in parallel before the sweep, when they
    // fit a bounded scratch (else each block is re-run inside the sweep)
    const size_t all_bytes =
        (size_t)n * ckpt_capacity * (SENS_CK_ATTEMPTS + 1) * SENS_STRIDE * sizeof(double);
    a.rec_all = nullptr;
    a.rep_count = nullptr;
    a.rep_first = nullptr;
    if (g_launch.adjoint_parallel_replay && all_bytes <= ADJOINT_REPLAY_BYTES) {
        void *ra, *rn, *rf;
        if ((rc = staging(*ds, 35, all_bytes, &ra)) ||
            (rc = staging(*ds, 36, (size_t)n * ckpt_capacity * sizeof(int32_t), &rn)) ||
            (rc = staging(*ds, 34, ((size_t)n + 2) * sizeof(int32_t), &rf)))
            return rc;
        a.rec_all = (double*)ra;
        a.rep_count = (int32_t*)rn;
        a.rep_first = (int32_t*)rf;
    }
    if ((rc = launch_sens_backward(a, st))) return rc;
    return S.finish();
}

int kete_b200_propagate_n_body_long(int64_t n, const double* pos, const double* vel, double jd0,
                                    double jd1, const double* planets, const double* nongrav,
                                    int batch_size, double* out_pos, double* out_vel,
                                    double* out_planets, int32_t* status, int on_device,
                                    void* stream) {
    if (n < 0 || batch_size < 1 || batch_size > 55)
        return set_error(KETE_B200_E_ARGUMENT, "need n >= 0 and a batch size of 1 to 55");
    if (n > 0 && (!pos || !vel || !out_pos || !out_vel || !status))
        return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (!std::isfinite(jd0) || !std::isfinite(jd1))
        return set_error(KETE_B200_E_ARGUMENT, "epochs must be finite");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    LongArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = n;
    a.pos = S.in(pos, 3 * (size_t)n);
    a.vel = S.in(vel, 3 * (size_t)n);
    a.jd0 = jd0;
    a.jd1 = jd1;
    a.nongrav = S.in(nongrav, 10 * (size_t)n);
    a.batch = batch_size;
    a.out_pos = S.out(out_pos, 3 * (size_t)n);
    a.out_vel = S.out(out_vel, 3 * (size_t)n);
    a.out_planets = S.out(out_planets, 54);
    a.status = S.out(status, (size_t)n);
    a.max_loops = g_launch.max_loops_long;
    if (planets) {
        a.planets = S.in(planets, 54);
    } else {
        // SpkCollection::try_get_state(id, jd0, 10, Equatorial) for the nine bodies
        // (mod.rs:166-176), on the device, into library scratch
        if (!g_eph.loaded) return set_error(KETE_B200_E_NO_EPHEMERIS, "no SPK loaded");
        static const int64_t ids[9] = {10, 1, 2, 3, 4, 5, 6, 7, 8};
        CenterChain ch;
        if ((rc = center_chain(10, ch))) return rc;
        void *pl = nullptr, *pst = nullptr, *pjd = nullptr;
        if ((rc = staging(*ds, 36, 54 * sizeof(double), &pl)) ||
            (rc = staging(*ds, 37, 9 * sizeof(int32_t), &pst)) ||
            (rc = staging(*ds, 38, sizeof(double), &pjd)))
            return rc;
        if ((rc = cuda_check(cudaMemcpyAsync(pjd, &a.jd0, sizeof(double), cudaMemcpyHostToDevice, st),
                             "copy epoch")))
            return rc;
        for (int k = 0; k < 9; ++k) {
            auto it = g_slot_of.find(ids[k]);
            if (it == g_slot_of.end())
                return set_error(KETE_B200_E_NO_EPHEMERIS,
                                 "Object (" + std::to_string(ids[k]) + ") does not have an SPK record");
            if ((rc = launch_spk_states(1, it->second, (const double*)pjd, ch, FRAME_EQUATORIAL,
                                        (double*)pl + 6 * k, (int32_t*)pst + k, st)))
                return rc;
        }
        a.planets = (const double*)pl;
        a.planet_status = (const int32_t*)pst;
        // the epoch copy reads a host stack value: wait for it before returning
        if ((rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize"))) return rc;
    }
    if (S.rc) return S.rc;
    if ((rc = launch_nbody_long(a, st))) return rc;
    return S.finish();
}

int kete_b200_fov_contains(int64_t n_vec, const double* vec, int64_t n_fov, const double* fov,
                           int64_t capacity, int32_t* out_fov, int32_t* out_idx,
                           int64_t* n_found, int on_device, void* stream) {
    if (n_vec < 0 || n_fov < 0 || capacity < 0 || !n_found)
        return set_error(KETE_B200_E_ARGUMENT, "negative size or null count");
    if (n_vec > 0 && !vec) return set_error(KETE_B200_E_ARGUMENT, "null direction array");
    if (n_fov > 0 && !fov) return set_error(KETE_B200_E_ARGUMENT, "null field table");
    if (capacity > 0 && (!out_fov || !out_idx)) return set_error(KETE_B200_E_ARGUMENT, "null output");
    if (n_vec > INT32_MAX || n_fov > INT32_MAX)
        return set_error(KETE_B200_E_ARGUMENT, "more than 2^31 directions or fields");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    *n_found = 0;
    if (n_vec == 0 || n_fov == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    const double* d_vec = S.in(vec, 3 * (size_t)n_vec);
    const double* d_fov = S.in(fov, (size_t)FOV_STRIDE * n_fov);
    int32_t* d_f = S.out(out_fov, (size_t)capacity);
    int32_t* d_i = S.out(out_idx, (size_t)capacity);
    if (S.rc) return S.rc;
    void* cnt = nullptr;
    if ((rc = staging(*ds, 35, sizeof(unsigned long long), &cnt))) return rc;
    if ((rc = cuda_check(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st), "clear counter")))
        return rc;
    if ((rc = launch_fov_contains(n_vec, d_vec, n_fov, d_fov, capacity, (unsigned long long*)cnt, d_f,
                                  d_i, st)))
        return rc;
    unsigned long long h = 0;
    if ((rc = cuda_check(cudaMemcpyAsync(&h, cnt, sizeof h, cudaMemcpyDeviceToHost, st), "read counter")))
        return rc;
    if ((rc = S.finish())) return rc;
    if ((rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize"))) return rc;
    *n_found = (int64_t)h;
    return 0;
}

int kete_b200_fov_check_visible(int64_t n_obj, const double* pos, const double* vel,
                                const double* jd, const uint8_t* valid, int64_t n_fov,
                                const double* fov, double dt_limit, int include_asteroids,
                                int64_t capacity, int32_t* out_fov, int32_t* out_obj,
                                double* out_state, int64_t* n_visible, int on_device,
                                void* stream) {
    if (n_obj < 0 || n_fov < 0 || capacity < 0 || !n_visible)
        return set_error(KETE_B200_E_ARGUMENT, "negative size or null count");
    if (n_obj > 0 && (!pos || !vel || !jd)) return set_error(KETE_B200_E_ARGUMENT, "null array");
    if (n_fov > 0 && !fov) return set_error(KETE_B200_E_ARGUMENT, "null field table");
    if (capacity > 0 && (!out_fov || !out_obj || !out_state))
        return set_error(KETE_B200_E_ARGUMENT, "null output");
    if (n_obj > INT32_MAX || n_fov > INT32_MAX)
        return set_error(KETE_B200_E_ARGUMENT, "more than 2^31 objects or fields");
    std::lock_guard<std::mutex> lk(g_mu);
    DevState* ds;
    int rc = ensure_device(ds);
    if (rc) return rc;
    *n_visible = 0;
    if (n_obj == 0 || n_fov == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    Stager S{*ds, st, on_device};
    FovArgs a;
    std::memset(&a, 0, sizeof a);
    a.n_obj = n_obj;
    a.pos = S.in(pos, 3 * (size_t)n_obj);
    a.vel = S.in(vel, 3 * (size_t)n_obj);
    a.jd = S.in(jd, (size_t)n_obj);
    a.valid = S.in(valid, (size_t)n_obj);
    a.n_fov = n_fov;
    a.fov = S.in(fov, (size_t)FOV_STRIDE * n_fov);
    a.dt_limit = dt_limit;
    a.capacity = capacity;
    a.out_fov = S.out(out_fov, (size_t)capacity);
    a.out_obj = S.out(out_obj, (size_t)capacity);
    a.out_state = S.out(out_state, 7 * (size_t)capacity);
    if (S.rc) return S.rc;
    // scratch: counters, the n-body candidate list and the screened-pair list (grown and
    // re-run on overflow)
    void* cnt = nullptr;
    if ((rc = staging(*ds, 20, 3 * sizeof(unsigned long long), &cnt))) return rc;
    a.counters = (unsigned long long*)cnt;
    const bool two_pass = g_launch.fov_form == 0;
    int64_t cand_cap = std::max<int64_t>(1024, n_obj / 16);
    int64_t pair_cap = std::max<int64_t>(4096, n_obj / 4);
    unsigned long long h[3] = {0, 0, 0};
    for (int attempt = 0; attempt < 3; ++attempt) {
        void *cf = nullptr, *co = nullptr, *pf = nullptr, *po = nullptr;
        if ((rc = staging(*ds, 21, (size_t)cand_cap * sizeof(int32_t), &cf))) return rc;
        if ((rc = staging(*ds, 22, (size_t)cand_cap * sizeof(int32_t), &co))) return rc;
        if (two_pass) {
            if ((rc = staging(*ds, 30, (size_t)pair_cap * sizeof(int32_t), &pf))) return rc;
            if ((rc = staging(*ds, 31, (size_t)pair_cap * sizeof(int32_t), &po))) return rc;
        }
        a.cand_fov = (int32_t*)cf;
        a.cand_obj = (int32_t*)co;
        a.cand_capacity = cand_cap;
        a.pair_fov = (int32_t*)pf;
        a.pair_obj = (int32_t*)po;
        a.pair_capacity = two_pass ? pair_cap : 0;
        if ((rc = cuda_check(cudaMemsetAsync(cnt, 0, 3 * sizeof(unsigned long long), st), "clear counters")))
            return rc;
        if ((rc = two_pass ? launch_fov_screen(a, st) : launch_fov_prefilter(a, st))) return rc;
        if ((rc = cuda_check(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, st), "read counters")))
            return rc;
        if ((rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize"))) return rc;
        if ((int64_t)h[1] <= cand_cap && (!two_pass || (int64_t)h[2] <= pair_cap)) break;
        cand_cap = std::max<int64_t>(cand_cap, (int64_t)h[1] + 1024);
        pair_cap = std::max<int64_t>(pair_cap, (int64_t)h[2] + 4096);
        if (attempt == 2) return set_error(KETE_B200_E_CUDA, "candidate list kept overflowing");
    }
    if (two_pass && (rc = launch_fov_pairs(a, (int64_t)h[2], st))) return rc;
    const int64_t m = (int64_t)h[1];
    if (m > 0) {
        // n-body branch (fov_like.rs:90-108): Radau every candidate to its field's epoch
        const int n_force = include_asteroids ? g_eph.n_force_all : g_eph.n_force_planets;
        if (!g_eph.loaded || n_force == 0)
            return set_error(KETE_B200_E_NO_EPHEMERIS, "the n-body FOV check needs a loaded SPK");
        void *gp, *gv, *g0, *g1, *op, *ov, *os;
        if ((rc = staging(*ds, 23, 3 * (size_t)m * sizeof(double), &gp)) ||
            (rc = staging(*ds, 24, 3 * (size_t)m * sizeof(double), &gv)) ||
            (rc = staging(*ds, 25, (size_t)m * sizeof(double), &g0)) ||
            (rc = staging(*ds, 26, (size_t)m * sizeof(double), &g1)) ||
            (rc = staging(*ds, 27, 3 * (size_t)m * sizeof(double), &op)) ||
            (rc = staging(*ds, 28, 3 * (size_t)m * sizeof(double), &ov)) ||
            (rc = staging(*ds, 29, (size_t)m * sizeof(int32_t), &os)))
            return rc;
        if ((rc = launch_fov_gather(a, m, (double*)gp, (double*)gv, (double*)g0, (double*)g1, st)))
            return rc;
        NBodyArgs nb;
        std::memset(&nb, 0, sizeof nb);
        if ((rc = center_chain(10, nb.chain))) return rc;
        nb.n = m;
        nb.pos = (double*)gp;
        nb.vel = (double*)gv;
        nb.jd0 = (double*)g0;
        nb.jd1 = (double*)g1;
        nb.frame = FRAME_ECLIPTIC;
        nb.n_force = n_force;
        nb.out_pos = (double*)op;
        nb.out_vel = (double*)ov;
        nb.status = (int32_t*)os;
        nb.max_loops = g_launch.max_loops;
        // one group per candidate, with a variant that carries the general ephemeris evaluation
        // (the warp-pooled kernels take only the objects inside the fast window)
        const int v = nodes_variant_for(g_launch.nodes_variant, nb.n_force);
        if ((rc = launch_nbody_nodes(nb, v >= 9 ? nodes_variant_for(7, nb.n_force) : v, 0, st)))
            return rc;
        if ((rc = launch_fov_finish(a, m, (double*)op, (double*)ov, (int32_t*)os, st))) return rc;
    }
    // the visible count after the last pass that emits (two-body pairs, n-body finish)
    if ((rc = cuda_check(cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, st), "read counters")))
        return rc;
    if ((rc = S.finish())) return rc;
    if ((rc = cuda_check(cudaStreamSynchronize(st), "stream synchronize"))) return rc;
    *n_visible = (int64_t)h[0];
    return 0;
}

int kete_b200_set_launch_config(int nodes_variant, int nodes_refill, int thread_block) {
    if (nodes_variant < 0 || nodes_variant > 10 || thread_block < 32 || thread_block > 1024 ||
        thread_block % 32)
        return set_error(KETE_B200_E_ARGUMENT, "bad launch configuration");
    std::lock_guard<std::mutex> lk(g_mu);
    g_launch.nodes_variant = nodes_variant;
    g_launch.nodes_refill = nodes_refill ? 1 : 0;
    g_launch.thread_block = thread_block;
    return 0;
}

int kete_b200_set_fov_form(int form) {
    if (form != 0 && form != 1) return set_error(KETE_B200_E_ARGUMENT, "field-check form is 0 or 1");
    std::lock_guard<std::mutex> lk(g_mu);
    g_launch.fov_form = form;
    return 0;
}

int kete_b200_set_sensitivity_form(int form) {
    if (form != 0 && form != 1) return set_error(KETE_B200_E_ARGUMENT, "sensitivity form is 0 or 1");
    std::lock_guard<std::mutex> lk(g_mu);
    g_launch.sens_form = form;
    return 0;
}

int kete_b200_set_adjoint_form(int form) {
    if (form != 0 && form != 1) return set_error(KETE_B200_E_ARGUMENT, "adjoint form is 0 or 1");
    std::lock_guard<std::mutex> lk(g_mu);
    g_launch.adjoint_parallel_replay = form == 0;
    return 0;
}

int kete_b200_set_step_limit(int64_t max_steps) {
    if (max_steps < 0 || max_steps > KETE_B200_STEP_LIMIT_MAX)
        return set_error(KETE_B200_E_ARGUMENT, "step limit out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    const LaunchConfig defaults;
    g_launch.max_loops = max_steps ? (int)max_steps : defaults.max_loops;
    g_launch.max_loops_long = max_steps ? (int)max_steps : defaults.max_loops_long;
    return 0;
}

int kete_b200_fp64_probe(int64_t iters, double* tflops, float* ms) {
    if (iters <= 0 || !tflops) return set_error(KETE_B200_E_ARGUMENT, "bad probe arguments");
    std::lock_guard<std::mutex> lk(g_mu);
    return fp64_probe(iters, tflops, ms);
}

}  // extern "C"
