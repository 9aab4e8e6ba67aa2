// CollisionDetector.hpp - header-only C++ facade over the C ABI (rtcd.h) with
// the method names of the upstream RTCD::CollisionDetector
// (RTCD/CollisionDetector/CollisionDetector.h:18-157) and robot wrapper
// (RTCD/CollisionDetector/CCRobotWrapper.h:12-70), so code written against the
// upstream call sequence
//     CollisionDetector cd(ctx, robot, scene);
//     cd.setupScene(scene); cd.setupOptix(); cd.setupRobot(robot); cd.buildSBT();
//     robot.prepareUpdateData(poses, n); cd.setNCheck(n); cd.check();
//     cd.downloadResult(result);
// ports by changing includes and constructors.  Errors become rtcd::Error
// exceptions on this side of the ABI.
#pragma once
#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../rtcd.h"

namespace rtcd {

struct Error : std::runtime_error {
    rtcd_status status;
    Error(rtcd_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check_status(rtcd_status s) {
    if (s == RTCD_OK) return;
    char buf[1024];
    rtcd_last_error(buf, sizeof(buf));
    throw Error(s, buf);
}

class Context {
public:
    explicit Context(int device = 0) { check_status(rtcd_context_create(device, &h_)); }
    ~Context() { rtcd_context_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    rtcd_ctx* get() const { return h_; }

private:
    rtcd_ctx* h_ = nullptr;
};

// Robot: chain + link meshes (+ spheres for the sweep detectors).  Holds the
// staged poses like the upstream CCWrappedRobot / CCRayRobot.
class Robot {
public:
    Robot(Context& ctx, const rtcd_robot_desc& desc) { check_status(rtcd_robot_create(ctx.get(), &desc, &h_)); }
    ~Robot() { rtcd_robot_destroy(h_); }
    Robot(const Robot&) = delete;
    Robot& operator=(const Robot&) = delete;
    rtcd_robot* get() const { return h_; }
    uint32_t dof() const { return dof_; }
    void setDof(uint32_t d) { dof_ = d; }

    // upstream CCWrappedRobot::prepareUpdateData(float* poses, size_t n)
    // (CCRobotWrapper.h:39-46): copies host poses ([n][dof], or all waypoints
    // of n trajectories with trajOffsets) for the next check().
    void prepareUpdateData(const float* poses, size_t n, const uint32_t* trajOffsets = nullptr) {
        trajOffsets_.clear();
        size_t rows = n;
        if (trajOffsets) {
            trajOffsets_.assign(trajOffsets, trajOffsets + n + 1);
            rows = trajOffsets[n];
        }
        poses_.assign(poses, poses + rows * dof_);
        n_ = n;
    }
    const std::vector<float>& poses() const { return poses_; }
    const std::vector<uint32_t>& trajOffsets() const { return trajOffsets_; }
    size_t staged() const { return n_; }

private:
    rtcd_robot* h_ = nullptr;
    uint32_t dof_ = 7;
    std::vector<float> poses_;
    std::vector<uint32_t> trajOffsets_;
    size_t n_ = 0;
};

class Scene {
public:
    Scene(Context& ctx, const std::vector<float>& verts, const std::vector<uint32_t>& tris,
          const std::vector<uint32_t>& obstacleTriOffsets) {
        check_status(rtcd_scene_create(ctx.get(), verts.data(), (uint32_t) (verts.size() / 3), tris.data(),
                                       (uint32_t) (tris.size() / 3),
                                       obstacleTriOffsets.empty() ? nullptr : obstacleTriOffsets.data(),
                                       obstacleTriOffsets.empty() ? 0u : (uint32_t) obstacleTriOffsets.size() - 1, &h_));
    }
    ~Scene() { rtcd_scene_destroy(h_); }
    Scene(const Scene&) = delete;
    Scene& operator=(const Scene&) = delete;
    rtcd_scene* get() const { return h_; }

private:
    rtcd_scene* h_ = nullptr;
};

// upstream LinkType values of the four detectors (RTCD/Meshes/meshTypes.h:37-48)
enum class LinkType { MESH, RAY_ONLINE, LINEAR_CURVE, QUADRATIC_CURVE };

inline rtcd_detector_kind to_kind(LinkType t) {
    switch (t) {
    case LinkType::MESH: return RTCD_OBS_TO_ROBOT;
    case LinkType::RAY_ONLINE: return RTCD_ROBOT_TO_OBS;
    case LinkType::LINEAR_CURVE: return RTCD_LINEAR_SWEEP;
    default: return RTCD_QUAD_SWEEP;
    }
}

template <LinkType TYPE>
class CollisionDetector {
public:
    CollisionDetector(Context& ctx, Robot& robot, Scene& scene) : ctx_(ctx), robot_(&robot), scene_(&scene) {}
    ~CollisionDetector() { rtcd_detector_destroy(det_); }
    CollisionDetector(const CollisionDetector&) = delete;
    CollisionDetector& operator=(const CollisionDetector&) = delete;

    void setupScene(Scene& s) { scene_ = &s; reset(); }
    void setupRobot(Robot& r) { robot_ = &r; reset(); }
    void setupOptix() {}  // nothing to compile: the kernels are built into the library
    void buildSBT() {
        if (!det_) check_status(rtcd_detector_create(ctx_.get(), to_kind(TYPE), robot_->get(), scene_->get(), nullptr, &det_));
    }
    void setNCheck(uint32_t n) { nCheck_ = n; }
    // The curve detectors follow the reference's semantics by default (its
    // loop edges counted where they enter a swept piece: RTCD_CHECK_SURFACE);
    // solid semantics (every obstacle edge within r of a sphere's path, plus
    // the start and end spheres of quadratic pieces) on request.
    void setSolidSweeps(bool solid) { solid_ = solid; }

    // Runs the staged query; upstream check() (CollisionDetector.h:422-471).
    void check() {
        buildSBT();
        const auto& q = robot_->poses();
        const auto& off = robot_->trajOffsets();
        uint32_t n = nCheck_ ? nCheck_ : (uint32_t) robot_->staged();
        flags_.assign(n, 0);
        counts_.assign(n, 0);
        const bool curve = TYPE == LinkType::LINEAR_CURVE || TYPE == LinkType::QUADRATIC_CURVE;
        const uint32_t sem = curve && !solid_ ? RTCD_CHECK_SURFACE : 0u;
        check_status(rtcd_check(det_, q.data(), off.empty() ? nullptr : off.data(), n, flags_.data(), nullptr,
                                counts_.data(), RTCD_CHECK_HOST_BUFFERS | RTCD_CHECK_COUNTS | sem, nullptr));
    }

    // Upstream downloadResult(std::vector<uint>&): per-pose (per-trajectory)
    // hit counts; nonzero means in collision.
    void downloadResult(std::vector<uint32_t>& result) const { result = counts_; }
    void downloadFlags(std::vector<uint8_t>& flags) const { flags = flags_; }
    void clearResult() { std::fill(counts_.begin(), counts_.end(), 0u); std::fill(flags_.begin(), flags_.end(), 0); }
    void resetGraph() {}
    rtcd_detector* get() const { return det_; }

private:
    void reset() {
        if (det_) rtcd_detector_destroy(det_);
        det_ = nullptr;
    }
    Context& ctx_;
    Robot* robot_;
    Scene* scene_;
    rtcd_detector* det_ = nullptr;
    uint32_t nCheck_ = 0;
    bool solid_ = false;
    std::vector<uint8_t> flags_;
    std::vector<uint32_t> counts_;
};

}  // namespace rtcd
