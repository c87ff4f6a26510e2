/*
 * bfm_io.hpp -- reader and writer of LeMonADE .bfm conformation files and of
 * .seeds files, for the pscbfm command-line simulator.
 *
 * LeMonADE's own reader (UpdaterReadBfmFile / FileImport / MoleculesRead) is
 * not part of the reference tree; the keys and the !mcs encoding follow the
 * reference's partial parser in src/pscbfm/mainColorBFM.cpp:135-286 and the
 * header lines its test script strips (testCorrectness.sh:78-114):
 *
 *   #!version=2.0                      comment / version line
 *   !number_of_monomers=N
 *   !box_x=L  !box_y=L  !box_z=L
 *   !periodic_x=1  !periodic_y=1  !periodic_z=1
 *   !set_of_bondvectors               lines "dx dy dz:id", id = byte used below
 *   !attributes                        lines "a-b:c" (1-based ranges)
 *   !bonds                             lines "a b"   (1-based, extra bonds)
 *   !mcs=AGE                           one frame: per line "x y z" then one
 *                                      space and one byte (bond id) per
 *                                      further monomer of the same chain
 *
 * Reading takes the last !mcs frame (READ_LAST_CONFIG_SAVE,
 * mainCUDASimulatorGPUScBFM_AB_Type.cpp:166).  Writing emits a header with the
 * 108 bond vectors (ids 17..124) and bonds that do not follow the chain
 * encoding, then appends frames.
 */
#pragma once

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace bfmio {

struct Conformation {
    uint32_t n = 0;
    uint64_t box[3] = {0, 0, 0};
    bool periodic[3] = {true, true, true};
    int64_t age = 0;
    std::vector<int32_t> xyz;                  /* 3n */
    std::vector<int32_t> attr;                 /* n */
    std::vector<std::vector<uint32_t>> nbr;    /* bond partners, 0-based, both directions */
    std::map<int, std::array<int, 3>> bondIds; /* id -> bond vector */
};

inline bool starts_with(const std::string &s, const char *p) { return s.compare(0, std::char_traits<char>::length(p), p) == 0; }

inline void add_bond(Conformation &c, uint32_t a, uint32_t b)
{
    if (a >= c.n || b >= c.n) throw std::runtime_error("bond partner out of range in .bfm file");
    c.nbr[a].push_back(b);
    c.nbr[b].push_back(a);
}

inline Conformation read_bfm(const std::string &path)
{
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<std::string> lines;
    for (std::string line; std::getline(f, line);) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        lines.push_back(line);
    }
    Conformation c;
    std::vector<std::pair<uint32_t, uint32_t>> bonds;
    size_t lastMcs = lines.size();
    for (size_t k = 0; k < lines.size(); ++k) {
        const std::string &l = lines[k];
        if (starts_with(l, "!number_of_monomers=")) c.n = (uint32_t)std::stoul(l.substr(20));
        else if (starts_with(l, "!box_x=")) c.box[0] = std::stoull(l.substr(7));
        else if (starts_with(l, "!box_y=")) c.box[1] = std::stoull(l.substr(7));
        else if (starts_with(l, "!box_z=")) c.box[2] = std::stoull(l.substr(7));
        else if (starts_with(l, "!periodic_x=")) c.periodic[0] = std::stoi(l.substr(12)) != 0;
        else if (starts_with(l, "!periodic_y=")) c.periodic[1] = std::stoi(l.substr(12)) != 0;
        else if (starts_with(l, "!periodic_z=")) c.periodic[2] = std::stoi(l.substr(12)) != 0;
        else if (starts_with(l, "!mcs")) lastMcs = k;
    }
    if (c.n == 0) throw std::runtime_error("!number_of_monomers missing in " + path);
    c.nbr.assign(c.n, {});
    c.attr.assign(c.n, 0);
    c.xyz.assign(3 * (size_t)c.n, 0);
    for (size_t k = 0; k < lines.size(); ++k) {
        const std::string &l = lines[k];
        if (l == "!set_of_bondvectors") {
            for (++k; k < lines.size() && !lines[k].empty() && lines[k][0] != '!'; ++k) {
                int dx, dy, dz, id;
                char colon;
                std::istringstream is(lines[k]);
                if (!(is >> dx >> dy >> dz >> colon >> id) || colon != ':') throw std::runtime_error("bad bond vector line: " + lines[k]);
                c.bondIds[id] = {dx, dy, dz};
            }
            --k;
        } else if (l == "!attributes") {
            for (++k; k < lines.size() && !lines[k].empty() && lines[k][0] != '!'; ++k) {
                unsigned a, b;
                int v;
                char dash, colon;
                std::istringstream is(lines[k]);
                if (!(is >> a >> dash >> b >> colon >> v) || a < 1 || b > c.n || a > b) throw std::runtime_error("bad attribute line: " + lines[k]);
                for (unsigned i = a; i <= b; ++i) c.attr[i - 1] = v;
            }
            --k;
        } else if (l == "!bonds") {
            for (++k; k < lines.size() && !lines[k].empty() && lines[k][0] != '!'; ++k) {
                unsigned a, b;
                std::istringstream is(lines[k]);
                if (!(is >> a >> b) || a < 1 || b < 1) throw std::runtime_error("bad bond line: " + lines[k]);
                bonds.emplace_back(a - 1, b - 1);
            }
            --k;
        }
    }
    if (lastMcs == lines.size()) throw std::invalid_argument("No conformation (starting with !mcs) found in " + path);
    {
        const std::string &h = lines[lastMcs];
        const size_t eq = h.find('=');
        c.age = eq == std::string::npos ? 0 : std::stoll(h.substr(eq + 1));
    }
    uint32_t m = 0;
    for (size_t k = lastMcs + 1; k < lines.size() && !lines[k].empty() && lines[k][0] != '!'; ++k) {
        const std::string &l = lines[k];
        std::istringstream is(l);
        long long x, y, z;
        if (!(is >> x >> y >> z)) throw std::runtime_error("bad monomer line in !mcs block");
        if (m >= c.n) throw std::runtime_error("more monomers in !mcs block than !number_of_monomers");
        c.xyz[3 * (size_t)m] = (int32_t)x;
        c.xyz[3 * (size_t)m + 1] = (int32_t)y;
        c.xyz[3 * (size_t)m + 2] = (int32_t)z;
        ++m;
        std::streampos p = is.tellg();
        if (p < 0) continue;
        size_t q = (size_t)p;
        if (q < l.size() && l[q] == ' ') ++q;
        for (; q < l.size(); ++q) {
            const int id = (unsigned char)l[q];
            auto it = c.bondIds.find(id);
            if (it == c.bondIds.end()) throw std::runtime_error("unknown bond vector id " + std::to_string(id));
            if (m >= c.n) throw std::runtime_error("more monomers in !mcs block than !number_of_monomers");
            x += it->second[0];
            y += it->second[1];
            z += it->second[2];
            c.xyz[3 * (size_t)m] = (int32_t)x;
            c.xyz[3 * (size_t)m + 1] = (int32_t)y;
            c.xyz[3 * (size_t)m + 2] = (int32_t)z;
            add_bond(c, m - 1, m);
            ++m;
        }
    }
    if (m != c.n) throw std::runtime_error("!mcs block holds " + std::to_string(m) + " monomers, expected " + std::to_string(c.n));
    for (auto &b : bonds) add_bond(c, b.first, b.second);
    return c;
}

/* the standard 108-vector set with ids 17..124 */
inline std::map<int, std::array<int, 3>> standard_bond_ids()
{
    std::map<int, std::array<int, 3>> out;
    int id = 17;
    for (int dx = -3; dx <= 3; ++dx)
        for (int dy = -3; dy <= 3; ++dy)
            for (int dz = -3; dz <= 3; ++dz) {
                int a[3] = {std::abs(dx), std::abs(dy), std::abs(dz)};
                std::sort(a, a + 3);
                const bool ok = (a[0] == 0 && a[1] == 0 && a[2] == 2) || (a[0] == 0 && a[1] == 1 && a[2] == 2) ||
                                (a[0] == 1 && a[1] == 1 && a[2] == 2) || (a[0] == 0 && a[1] == 0 && a[2] == 3) ||
                                (a[0] == 0 && a[1] == 1 && a[2] == 3) || (a[0] == 1 && a[1] == 2 && a[2] == 2);
                if (ok) out[id++] = {dx, dy, dz};
            }
    return out;
}

inline void write_header(const std::string &path, const Conformation &c, const std::map<int, std::array<int, 3>> &ids)
{
    std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("cannot write " + path);
    f << "#!version=2.0\n";
    f << "!number_of_monomers=" << c.n << "\n";
    f << "!box_x=" << c.box[0] << "\n!box_y=" << c.box[1] << "\n!box_z=" << c.box[2] << "\n";
    f << "!periodic_x=" << (int)c.periodic[0] << "\n!periodic_y=" << (int)c.periodic[1] << "\n!periodic_z=" << (int)c.periodic[2] << "\n";
    f << "!set_of_bondvectors\n";
    for (auto &kv : ids) f << kv.second[0] << " " << kv.second[1] << " " << kv.second[2] << ":" << kv.first << "\n";
    f << "\n!attributes\n";
    for (uint32_t i = 0; i < c.n;) {
        uint32_t j = i;
        while (j + 1 < c.n && c.attr[j + 1] == c.attr[i]) ++j;
        f << i + 1 << "-" << j + 1 << ":" << c.attr[i] << "\n";
        i = j + 1;
    }
    f << "\n!bonds\n";
    for (uint32_t i = 0; i < c.n; ++i)
        for (uint32_t k : c.nbr[i])
            if (k > i && k != i + 1) f << i + 1 << " " << k + 1 << "\n";
    f << "\n";
}

/* one !mcs frame; consecutive bonded monomers (i, i+1) are chain-encoded */
inline void append_frame(const std::string &path, const Conformation &c, const std::map<int, std::array<int, 3>> &ids)
{
    std::map<std::array<int, 3>, int> inv;
    for (auto &kv : ids) inv[kv.second] = kv.first;
    std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::app);
    if (!f) throw std::runtime_error("cannot append to " + path);
    f << "!mcs=" << c.age << "\n";
    for (uint32_t i = 0; i < c.n;) {
        f << c.xyz[3 * (size_t)i] << " " << c.xyz[3 * (size_t)i + 1] << " " << c.xyz[3 * (size_t)i + 2];
        uint32_t j = i;
        std::string chain;
        while (j + 1 < c.n) {
            bool bonded = false;
            for (uint32_t k : c.nbr[j])
                if (k == j + 1) bonded = true;
            if (!bonded) break;
            const std::array<int, 3> v = {c.xyz[3 * (size_t)(j + 1)] - c.xyz[3 * (size_t)j],
                                          c.xyz[3 * (size_t)(j + 1) + 1] - c.xyz[3 * (size_t)j + 1],
                                          c.xyz[3 * (size_t)(j + 1) + 2] - c.xyz[3 * (size_t)j + 2]};
            auto it = inv.find(v);
            if (it == inv.end()) break; /* not a set vector: the bond goes to !bonds */
            chain.push_back((char)it->second);
            ++j;
        }
        if (!chain.empty()) f << " " << chain;
        f << "\n";
        i = j + 1;
    }
    f << "\n";
}

/* .seeds: whitespace-separated unsigned 32-bit integers; at least 250 */
inline std::vector<uint32_t> read_seeds(const std::string &path)
{
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::vector<uint32_t> w;
    unsigned long long v;
    while (f >> v) w.push_back((uint32_t)v);
    if (w.size() < 250) throw std::runtime_error(".seeds file needs at least 250 values, got " + std::to_string(w.size()));
    return w;
}

} // namespace bfmio
