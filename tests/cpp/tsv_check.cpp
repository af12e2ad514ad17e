// tsv snapshots through include/grasph2_b200.hpp, for the byte-exactness test against GraSPH2's own
// writer and reader (tests/test_io_reference.py).
//   tsv_check write <dir/> <prefix> <start_time> <time> <n> <in.bin>
//       in.bin: float32 pos[3n], mass[n], vel[3n], density[n]; writes <dir/><prefix><start>_<time>.tsv
//       with the adapter's snapshotFileName + printTextFile and prints the file name
//   tsv_check read <file.tsv> <out.bin>
//       reads the file with readTextFile and writes n (int64) then the same four float32 arrays
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "grasph2_b200.hpp"

int main(int argc, char** argv) {
    const std::string mode = argc > 1 ? argv[1] : "";
    try {
        if (mode == "write" && argc == 8) {
            const int64_t n = std::stoll(argv[6]);
            gsph::HostParticleBuffer h(static_cast<size_t>(n));
            std::ifstream in(argv[7], std::ios::binary);
            in.read(reinterpret_cast<char*>(h.pos.data()), 3 * n * sizeof(float));
            in.read(reinterpret_cast<char*>(h.mass.data()), n * sizeof(float));
            in.read(reinterpret_cast<char*>(h.vel.data()), 3 * n * sizeof(float));
            in.read(reinterpret_cast<char*>(h.density.data()), n * sizeof(float));
            if (!in) throw std::runtime_error("short input");
            const std::string name = gsph::snapshotFileName(argv[2], argv[3], argv[4], std::stof(argv[5]));
            gsph::printTextFile(h, name);
            std::cout << name << "\n";
            return 0;
        }
        if (mode == "read" && argc == 4) {
            const gsph::HostParticleBuffer h = gsph::readTextFile(argv[2]);
            const int64_t n = static_cast<int64_t>(h.size());
            std::ofstream out(argv[3], std::ios::binary);
            out.write(reinterpret_cast<const char*>(&n), sizeof n);
            out.write(reinterpret_cast<const char*>(h.pos.data()), 3 * n * sizeof(float));
            out.write(reinterpret_cast<const char*>(h.mass.data()), n * sizeof(float));
            out.write(reinterpret_cast<const char*>(h.vel.data()), 3 * n * sizeof(float));
            out.write(reinterpret_cast<const char*>(h.density.data()), n * sizeof(float));
            return out ? 0 : 1;
        }
    } catch (const std::exception& e) {
        std::cerr << e.what() << "\n";
        return 1;
    }
    std::cerr << "usage: tsv_check write <dir/> <prefix> <start> <time> <n> <in.bin> | read <file> <out.bin>\n";
    return 2;
}
