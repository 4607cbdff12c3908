// A space-time caller of TerraNNI's nni:: interface, the way binRun
// (terranni.cpp:394-426) drives it: one work package, performNNI for every
// time from t_start to t_end on the same time-sorted point stream, then
// clearRenderbuffers.
//
// usage: nni_shim_time_demo <points.bin> <out_prefix> <ncols> <nrows> <cell_m> <query_radius_m>
//                           <time_radius> <t_start> <t_end> <delta: 1|0>
// points.bin holds raw nni::Point4D records sorted by time; each time t
// writes raw nni::OutPoint records to <out_prefix><t>.bin and prints
// "t <t> pos <stream position after the call>".
#include <cstdio>
#include <cstdlib>
#include <string>

#include <nni/nni.h>

int main(int argc, char** argv) {
    if (argc != 11) {
        std::fprintf(stderr, "usage: %s points.bin out_prefix ncols nrows cell_m qr time_radius t0 t1 delta\n", argv[0]);
        return 64;
    }
    nni::Settings s{};
    s.scale = 1;
    s.cell_size = (float)std::atof(argv[5]);
    s.ncols = std::atoi(argv[3]);
    s.nrows = std::atoi(argv[4]);
    s.query_radius = std::atof(argv[6]);
    s.site_radius = (float)s.query_radius;
    nni::WorkPackage wp{};
    wp.ncols = s.ncols;
    wp.nrows = s.nrows;
    const float tr = (float)std::atof(argv[7]);
    const int t0 = std::atoi(argv[8]), t1 = std::atoi(argv[9]);
    const bool delta = std::atoi(argv[10]) != 0;
    try {
        nni::init(s);
        nni::setupRun(wp);
        tpie::ami::stream<nni::Point4D> vec(argv[1], tpie::ami::READ_STREAM);
        vec.persist(tpie::ami::PERSIST_DELETE);   // leave the input file as it is
        vec.seek(0);
        for (int t = t0; t <= t1; ++t) {
            const std::string name = std::string(argv[2]) + std::to_string(t) + ".bin";
            tpie::ami::stream<nni::OutPoint> out(name, tpie::ami::WRITE_STREAM);
            nni::performNNI(wp, out, vec, tr, (float)t, delta);
            std::printf("t %d pos %lld\n", t, (long long)vec.tell());
        }
        nni::clearRenderbuffers();
        nni::cleanup();
    } catch (const nni::Error& e) {
        std::fprintf(stderr, "nni::Error %d: %s\n", (int)e.status, e.what());
        return (int)e.status;
    }
    return 0;
}
