// Firing-level decoder for LVXR recordings, on the host (lvxr.py read_firings :189-260; the datagram format of
// record.rs and point.rs): every firing with its exact time on the recording's time base, the empty ones
// included, so real recordings can be replayed through the pipeline.
//
// The decode follows lvxr.py step by step: the datagram walk (a truncated last datagram ends it), point packets
// of known layout, the time base over every point packet (reset when the clock goes backwards, shifted over a
// forward jump of a second or more), whole packets only (the Mid-40 dual profile: exactly 100 plain records, two
// returns per firing), records decoded per layout, firings ordered stably by time after the reference's grouping
// (data type, then datagram length, then file order), a cartesian firing's direction taken from its first return.
// Cartesian coordinates are exact (integer millimetres times 1e-3 in float32); spherical ones use float32 sin / cos
// of the reference's float32 angles, within an ulp or two of numpy's.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "lw_common.cuh"

using lw::set_error;

struct lw_lvxr {
    int64_t n = 0;
    int32_t R = 1, dev = 0, profile = 0;
    double interval = 0.0;
    std::vector<double> t;
    std::vector<float> xyz, dir;
    std::vector<uint8_t> refl, tag, valid;
};

namespace {

struct Layout {
    int size, R;
    bool sph;
};

bool layout_of(int d, Layout& L) {  // lvxr.py LAYOUTS :26-27
    switch (d) {
        case 0: L = {13, 1, false}; return true;
        case 1: L = {9, 1, true}; return true;
        case 2: L = {14, 1, false}; return true;
        case 3: L = {10, 1, true}; return true;
        case 4: L = {28, 2, false}; return true;
        case 5: L = {16, 2, true}; return true;
        case 7: L = {42, 3, false}; return true;
        case 8: L = {22, 3, true}; return true;
        default: return false;
    }
}

uint64_t rd_u(const uint8_t* p, int nbytes) {
    uint64_t v = 0;
    for (int j = 0; j < nbytes; ++j) v |= (uint64_t)p[j] << (8 * j);
    return v;
}

int32_t rd_i32(const uint8_t* p) { return (int32_t)(uint32_t)rd_u(p, 4); }

constexpr int HEADER_LEN = 18;
constexpr int64_t CLOCK_JUMP_NS = 1000000000LL;
constexpr int MID40_DUAL_RECORDS = 100;

struct Packet {
    int64_t off, len, records, t;
    int dtype, index;
};

// One record's returns into xyz [R*3], refl, tag; the direction of a spherical record into dir (lvxr.py _decode).
void decode_record(const uint8_t* r, int dtype, float* xyz, uint8_t* refl, uint8_t* tag, float* dir) {
    const float mm = 1e-3f;
    auto cart = [&](const uint8_t* p, int k) {
        xyz[3 * k + 0] = (float)rd_i32(p) * mm;
        xyz[3 * k + 1] = (float)rd_i32(p + 4) * mm;
        xyz[3 * k + 2] = (float)rd_i32(p + 8) * mm;
    };
    auto spherical = [&](uint32_t depth, uint16_t theta, uint16_t phi, int k) {
        const float d2r = 3.14159265358979323846f / 180.0f;  // numpy's float32 radians
        const float th = ((float)theta * 0.01f) * d2r, ph = ((float)phi * 0.01f) * d2r;
        const float st = std::sin(th);
        const float u[3] = {st * std::cos(ph), st * std::sin(ph), std::cos(th)};
        const float dm = (float)depth * mm;
        for (int c = 0; c < 3; ++c) {
            xyz[3 * k + c] = u[c] * dm;
            dir[c] = u[c];
        }
    };
    switch (dtype) {
        case 0: cart(r, 0); refl[0] = r[12]; break;
        case 2: cart(r, 0); refl[0] = r[12]; tag[0] = r[13]; break;
        case 1: spherical((uint32_t)rd_u(r, 4), (uint16_t)rd_u(r + 4, 2), (uint16_t)rd_u(r + 6, 2), 0); refl[0] = r[8]; break;
        case 3:
            spherical((uint32_t)rd_u(r, 4), (uint16_t)rd_u(r + 4, 2), (uint16_t)rd_u(r + 6, 2), 0);
            refl[0] = r[8];
            tag[0] = r[9];
            break;
        case 4:
        case 7:
            for (int k = 0; k < (dtype == 4 ? 2 : 3); ++k) {
                cart(r + 14 * k, k);
                refl[k] = r[14 * k + 12];
                tag[k] = r[14 * k + 13];
            }
            break;
        default: {  // 5, 8: one direction, R (depth, reflectivity, tag)
            const uint16_t theta = (uint16_t)rd_u(r, 2), phi = (uint16_t)rd_u(r + 2, 2);
            for (int k = 0; k < (dtype == 5 ? 2 : 3); ++k) {
                const uint8_t* b = r + 4 + 6 * k;
                spherical((uint32_t)rd_u(b, 4), theta, phi, k);
                refl[k] = b[4];
                tag[k] = b[5];
            }
        }
    }
}

}  // namespace

extern "C" {

int lw_lvxr_decode(const uint8_t* data, int64_t size, lw_lvxr** out) {
    if (!data || !out || size < 0) return set_error(LW_EINVAL, "lw_lvxr_decode: bad arguments");
    *out = nullptr;
    int dev, profile;
    int64_t off;
    if (size >= 7 && std::memcmp(data, "LVXR1\n", 6) == 0) {
        dev = data[6];
        profile = 0;
        off = 7;
    } else if (size >= 8 && std::memcmp(data, "LVXR2\n", 6) == 0) {
        dev = data[6];
        profile = data[7];
        off = 8;
    } else {
        return set_error(LW_EINVAL, "lw_lvxr_decode: not an LVXR recording");
    }
    const bool dual = profile == 1;
    const int64_t interval = (dev == 2 || dev == 3 || dev == 7) ? 4167 : 10000;
    // the datagrams: host_ns u64, len u16, datagram; a truncated last one ends the walk
    std::vector<Packet> pk;
    int index = 0;
    while (off + 10 <= size) {
        const int64_t ln = (int64_t)data[off + 8] | ((int64_t)data[off + 9] << 8);
        if (off + 10 + ln > size) break;
        const int64_t o = off + 10;
        Layout L;
        if (ln >= HEADER_LEN && layout_of(data[o + 9], L)) {
            Packet p{o, ln, (ln - HEADER_LEN) / L.size, 0, data[o + 9], index};
            uint64_t ts = rd_u(data + o + 10, 8);
            if (data[o + 8] == 3) ts = ((uint64_t)data[o + 13] * 3600000000ULL + rd_u(data + o + 14, 4)) * 1000ULL;  // GPS
            p.t = (int64_t)ts;
            pk.push_back(p);
        }
        ++index;
        off += 10 + ln;
    }
    // the time base over every point packet, malformed ones included (lvxr.py _time_base :112-132)
    {
        bool have_base = false, have_exp = false;
        int64_t base = 0, expected = 0;
        for (Packet& p : pk) {
            const int64_t t = p.t;
            const int64_t span = (dual ? p.records / 2 : p.records) * interval;
            if (!have_base || t < base) {
                base = t;
                have_base = true;
                have_exp = false;
            }
            if (have_exp && span > 0 && t > expected + span / 2) {
                const int64_t gap = t - expected;
                if (gap >= CLOCK_JUMP_NS) base += gap;
            }
            expected = t + span;
            have_exp = true;
            p.t = t - base;
        }
    }
    // whole packets only, grouped by data type, then datagram length, then file order
    std::vector<Packet> keep;
    for (const Packet& p : pk) {
        Layout L;
        layout_of(p.dtype, L);
        bool whole = (p.len - HEADER_LEN) == p.records * L.size;
        if (dual) whole = whole && (p.dtype == 0 || p.dtype == 1) && p.records == MID40_DUAL_RECORDS;
        if (whole) keep.push_back(p);
    }
    if (keep.empty()) return set_error(LW_EINVAL, "lw_lvxr_decode: no point packets");
    std::stable_sort(keep.begin(), keep.end(), [](const Packet& a, const Packet& b) {
        if (a.dtype != b.dtype) return a.dtype < b.dtype;
        if (a.len != b.len) return a.len < b.len;
        return a.index < b.index;
    });
    int R = dual ? 2 : 1;
    int64_t n = 0;
    for (const Packet& p : keep) {
        Layout L;
        layout_of(p.dtype, L);
        R = std::max(R, L.R);
        n += dual ? p.records / 2 : p.records;
    }
    lw_lvxr* rec = new lw_lvxr();
    rec->n = n;
    rec->R = R;
    rec->dev = dev;
    rec->profile = profile;
    rec->interval = (double)interval * 1e-9;
    std::vector<double> t(n);
    std::vector<float> xyz((size_t)n * R * 3, 0.0f), dir((size_t)n * 3, std::nanf(""));
    std::vector<uint8_t> refl((size_t)n * R, 0), tag((size_t)n * R, 0);
    int64_t f = 0;
    for (const Packet& p : keep) {
        Layout L;
        layout_of(p.dtype, L);
        const uint8_t* body = data + p.off + HEADER_LEN;
        if (dual) {
            // plain records in pairs: the two returns of one firing; its direction is the first record's
            for (int64_t i = 0; i < p.records / 2; ++i, ++f) {
                t[f] = (double)(p.t + i * interval) * 1e-9;
                float d0[3], d1[3];
                decode_record(body + (2 * i) * L.size, p.dtype, &xyz[(f * R + 0) * 3], &refl[f * R + 0], &tag[f * R + 0], d0);
                decode_record(body + (2 * i + 1) * L.size, p.dtype, &xyz[(f * R + 1) * 3], &refl[f * R + 1], &tag[f * R + 1], d1);
                if (L.sph)
                    for (int c = 0; c < 3; ++c) dir[3 * f + c] = d0[c];
            }
        } else {
            for (int64_t i = 0; i < p.records; ++i, ++f) {
                t[f] = (double)(p.t + i * interval) * 1e-9;
                float d[3];
                decode_record(body + i * L.size, p.dtype, &xyz[f * R * 3], &refl[f * R], &tag[f * R], d);
                if (L.sph)
                    for (int c = 0; c < 3; ++c) dir[3 * f + c] = d[c];
            }
        }
    }
    // a return is valid when it has coordinates; an empty cartesian firing's direction is its first return's
    std::vector<uint8_t> valid((size_t)n * R, 0);
    for (int64_t i = 0; i < n; ++i) {
        int first = -1;
        for (int r = 0; r < R; ++r) {
            const float* v = &xyz[(i * R + r) * 3];
            valid[i * R + r] = (v[0] != 0.0f || v[1] != 0.0f || v[2] != 0.0f) ? 1 : 0;
            if (valid[i * R + r] && first < 0) first = r;
        }
        if (std::isnan(dir[3 * i]) && first >= 0) {
            const float* v = &xyz[(i * R + first) * 3];
            const float nrm = std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
            for (int c = 0; c < 3; ++c) dir[3 * i + c] = v[c] / nrm;
        }
    }
    // time order, stable
    std::vector<int64_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return t[a] < t[b]; });
    rec->t.resize(n);
    rec->xyz.resize((size_t)n * R * 3);
    rec->dir.resize((size_t)n * 3);
    rec->refl.resize((size_t)n * R);
    rec->tag.resize((size_t)n * R);
    rec->valid.resize((size_t)n * R);
    for (int64_t i = 0; i < n; ++i) {
        const int64_t s = order[i];
        rec->t[i] = t[s];
        std::memcpy(&rec->xyz[(size_t)i * R * 3], &xyz[(size_t)s * R * 3], sizeof(float) * R * 3);
        std::memcpy(&rec->dir[(size_t)i * 3], &dir[(size_t)s * 3], sizeof(float) * 3);
        std::memcpy(&rec->refl[(size_t)i * R], &refl[(size_t)s * R], R);
        std::memcpy(&rec->tag[(size_t)i * R], &tag[(size_t)s * R], R);
        std::memcpy(&rec->valid[(size_t)i * R], &valid[(size_t)s * R], R);
    }
    *out = rec;
    return LW_OK;
}

int lw_lvxr_info(const lw_lvxr* r, int64_t* n_firings, int32_t* returns, int32_t* dev_type, int32_t* profile,
                 double* interval_s) {
    if (!r || !n_firings || !returns || !dev_type || !profile || !interval_s)
        return set_error(LW_EINVAL, "lw_lvxr_info: bad arguments");
    *n_firings = r->n;
    *returns = r->R;
    *dev_type = r->dev;
    *profile = r->profile;
    *interval_s = r->interval;
    return LW_OK;
}

int lw_lvxr_copy(const lw_lvxr* r, double* t, float* xyz, uint8_t* refl, uint8_t* tag, uint8_t* valid,
                 float* direction) {
    if (!r || !t || !xyz || !refl || !tag || !valid || !direction) return set_error(LW_EINVAL, "lw_lvxr_copy: bad arguments");
    const size_t n = (size_t)r->n, R = (size_t)r->R;
    std::memcpy(t, r->t.data(), sizeof(double) * n);
    std::memcpy(xyz, r->xyz.data(), sizeof(float) * n * R * 3);
    std::memcpy(refl, r->refl.data(), n * R);
    std::memcpy(tag, r->tag.data(), n * R);
    std::memcpy(valid, r->valid.data(), n * R);
    std::memcpy(direction, r->dir.data(), sizeof(float) * n * 3);
    return LW_OK;
}

void lw_lvxr_free(lw_lvxr* r) { delete r; }

}  // extern "C"
