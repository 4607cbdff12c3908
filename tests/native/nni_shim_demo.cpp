// A caller written against TerraNNI's nni:: interface (nni.h:83-97), the way
// binRun (terranni.cpp:394-426) drives it, built against include/nni/nni.h
// and libdnni.so instead of the GL library.
//
// usage: nni_shim_demo <points.bin> <out.bin> <ncols> <nrows> <cell_m> <origin_x> <origin_y>
//                      <grid_origin_x> <grid_origin_y> <total_ncols> <total_nrows> <query_radius_m>
//                      [<scale> <site_radius_m> <pointMin> <multiplier>]
// The four optional arguments switch the shim to the reference's default
// semantics (nni::setCompatMode) with those settings.  points.bin holds raw
// nni::Point4D records; out.bin receives raw nni::OutPoint records.  Exit
// status: 0, or the engine status of an nni::Error.
#include <cstdio>
#include <cstdlib>

#include <nni/nni.h>

int main(int argc, char** argv) {
    if (argc != 13 && argc != 17) {
        std::fprintf(stderr, "usage: %s points.bin out.bin ncols nrows cell_m ox oy gox goy total_ncols total_nrows qr\n",
                     argv[0]);
        return 64;
    }
    nni::Settings s{};
    s.scale = 1;
    s.cell_size = (float)std::atof(argv[5]);
    s.ncols = std::atoi(argv[10]);
    s.nrows = std::atoi(argv[11]);
    s.query_radius = std::atof(argv[12]);
    s.site_radius = (float)s.query_radius;
    if (argc == 17) {
        s.scale = std::atoi(argv[13]);
        s.site_radius = (float)std::atof(argv[14]);
        s.pointMin = std::atoi(argv[15]);
        s.multiplier = std::atoi(argv[16]);
        nni::setCompatMode(true);
    }
    nni::WorkPackage wp{};
    wp.ncols = std::atoi(argv[3]);
    wp.nrows = std::atoi(argv[4]);
    wp.origin_x = (float)std::atof(argv[6]);
    wp.origin_y = (float)std::atof(argv[7]);
    wp.grid_origin_x = (float)std::atof(argv[8]);
    wp.grid_origin_y = (float)std::atof(argv[9]);
    try {
        nni::init(s);
        nni::setupRun(wp);
        {
            tpie::ami::stream<nni::Point4D> vec(argv[1], tpie::ami::READ_STREAM);
            vec.persist(tpie::ami::PERSIST_DELETE);   // leave the input file as it is
            tpie::ami::stream<nni::OutPoint> out(argv[2], tpie::ami::WRITE_STREAM);
            vec.seek(0);
            nni::performNNI(wp, out, vec, 0.0f, 0.0f, false);
            nni::clearRenderbuffers();
            std::printf("outpoints %lld, stream position %lld of %lld\n", (long long)out.stream_len(),
                        (long long)vec.tell(), (long long)vec.stream_len());
        }
        nni::printTimes();
        nni::cleanup();
    } catch (const nni::Error& e) {
        std::fprintf(stderr, "nni::Error %d: %s\n", (int)e.status, e.what());
        return (int)e.status;
    }
    return 0;
}
