// Runs the host planner (orrery_b200/csrc/plan.cpp) on the lattices of a case
// file, for builds under ThreadSanitizer and AddressSanitizer + UBSan.  The
// cases are large enough (at least 2^20 cells) for validation and planning to
// run on several host threads.  Per case it prints the refusal text, or the
// node counts and FNV-1a digests of every table the plan holds, so that two
// differently instrumented builds and the library can be compared.
//
// Case file: repeated records of
//   uint32 config_bytes, orr_lbm3d_config, uint64 cells, uint8 solid[cells],
//   uint8 has_distance, double distance[cells] (when has_distance)
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "plan.h"

namespace {

uint64_t fnv1a(const void* data, std::size_t bytes, uint64_t h = 1469598103934665603ull) {
    const auto* p = static_cast<const unsigned char*>(data);
    for (std::size_t i = 0; i < bytes; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

template <class V> uint64_t digest(const V& v) {
    return fnv1a(v.data(), v.size() * sizeof(typename V::value_type));
}

template <class T> bool read(std::ifstream& in, T& v) {
    return static_cast<bool>(in.read(reinterpret_cast<char*>(&v), sizeof v));
}

} // namespace

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s <case file>\n", argv[0]);
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    for (int k = 0;; ++k) {
        uint32_t config_bytes = 0;
        if (!read(in, config_bytes)) {
            break;
        }
        if (config_bytes != sizeof(orr_lbm3d_config)) {
            std::fprintf(stderr, "case %d: config record of %u bytes, expected %zu\n", k, config_bytes,
                         sizeof(orr_lbm3d_config));
            return 3;
        }
        orr_lbm3d_config c{};
        uint64_t cells = 0;
        uint8_t has_distance = 0;
        if (!read(in, c) || !read(in, cells)) {
            return 4;
        }
        std::vector<uint8_t> solid(cells);
        std::vector<double> distance;
        in.read(reinterpret_cast<char*>(solid.data()), static_cast<std::streamsize>(cells));
        if (!read(in, has_distance)) {
            return 4;
        }
        if (has_distance) {
            distance.resize(cells);
            in.read(reinterpret_cast<char*>(distance.data()), static_cast<std::streamsize>(cells * sizeof(double)));
        }
        if (!in) {
            return 4;
        }
        const double* dist = has_distance ? distance.data() : nullptr;
        const std::string problem = orr::problem3d(c, solid.data(), dist, ORR_STORAGE_F32, false);
        if (!problem.empty()) {
            std::printf("case %d refused %s\n", k, problem.c_str());
            continue;
        }
        const orr::Plan3D p = orr::plan3d(c, solid.data(), dist);
        uint64_t links = fnv1a(p.link_cell.data(), p.link_cell.size() * sizeof(uint32_t));
        links = fnv1a(p.link_dir.data(), p.link_dir.size() * sizeof(uint32_t), links);
        links = fnv1a(p.link_q.data(), p.link_q.size() * sizeof(double), links);
        std::printf("case %d fluid %zu general %zu links %zu links_digest %016llx cls %016llx nmask %016llx "
                    "nslot %016llx wall_q %016llx\n",
                    k, p.fluid, p.general, p.link_cell.size(), static_cast<unsigned long long>(links),
                    static_cast<unsigned long long>(digest(p.cls)), static_cast<unsigned long long>(digest(p.nmask)),
                    static_cast<unsigned long long>(digest(p.nslot)), static_cast<unsigned long long>(digest(p.wall_q)));
    }
    std::printf("ok\n");
    return 0;
}
