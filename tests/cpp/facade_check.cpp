// Drives the detector through the C++ facade with the upstream call sequence
// (RTCD/Demo/DemoCollisionDetectorDisc.cpp:56-76) on a one-triangle scene and
// a two-link toy robot, then prints "flags:" and "counts:" lines for the test
// to check.  Build: g++ -std=c++17 -I include tests/cpp/facade_check.cpp
//                   -L rtcollisiondetection_b200 -lrtcd_b200
#include <cstdio>
#include <vector>

#include "rtcd/CollisionDetector.hpp"

int main() {
    using namespace rtcd;
    try {
        Context ctx(0);
        // one revolute joint about z; link 1 is a flat square at height 0.5 spanning x in [0.2, 0.6]
        float base[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
        float cm[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0};
        float sm[12] = {0, -1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0};
        float om[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0};
        std::vector<float> lv = {-0.01f, -0.01f, 0.f, 0.01f, -0.01f, 0.f, 0.f, 0.01f, 0.f,           // link 0: tiny
                                 0.2f, -0.2f, 0.5f, 0.6f, -0.2f, 0.5f, 0.6f, 0.2f, 0.5f, 0.2f, 0.2f, 0.5f};
        std::vector<uint32_t> lvo = {0, 3, 7};
        std::vector<uint32_t> lt = {0, 1, 2, 0, 1, 2, 0, 2, 3};
        std::vector<uint32_t> lto = {0, 1, 3};
        rtcd_robot_desc d{};
        d.dof = 1; d.base_tf = base; d.cos_mask = cm; d.sin_mask = sm; d.one_mask = om;
        d.link_verts = lv.data(); d.link_vert_offsets = lvo.data(); d.link_tris = lt.data(); d.link_tri_offsets = lto.data();
        d.skip_base = 1;
        Robot robot(ctx, d);
        robot.setDof(1);
        // an upright wall crossing the plane z = 0.5 along x = 0.4, y in [-1, 1]
        std::vector<float> sv = {0.4f, -1.f, 0.f, 0.4f, 1.f, 0.f, 0.4f, 0.f, 1.f};
        std::vector<uint32_t> st = {0, 1, 2};
        Scene scene(ctx, sv, st, {0, 1});
        CollisionDetector<LinkType::RAY_ONLINE> cd(ctx, robot, scene);
        cd.setupScene(scene);
        cd.setupOptix();
        cd.setupRobot(robot);
        cd.buildSBT();
        std::vector<float> q = {0.0f, 3.14159f};  // facing the wall, facing away
        robot.prepareUpdateData(q.data(), 2);
        cd.setNCheck(2);
        cd.check();
        std::vector<uint32_t> counts;
        std::vector<uint8_t> flags;
        cd.downloadResult(counts);
        cd.downloadFlags(flags);
        std::printf("flags: %d %d\ncounts: %u %u\n", flags[0], flags[1], counts[0], counts[1]);
        return 0;
    } catch (const rtcd::Error& e) {
        std::fprintf(stderr, "rtcd error %d: %s\n", (int) e.status, e.what());
        return 2;
    }
}
