// cublox::OccupancyGrid drop-in over the cublox_b200 C ABI (sm_100a).
//
// Same class names, signatures, defaults and error behaviour as the
// reference's include/cublox/OccupancyGrid.hpp:29-169 and
// include/cublox/Grid.hpp:22-57: construction throws std::runtime_error on a
// CUDA failure or an int32 voxel-count overflow, degenerate inputs are silent
// no-ops, fetchOccupancyAround returns a std::vector<OccupancySample>, and the
// public Grid members (config_, origin_i_, ...) are kept current.  Header
// only; link with libcublox_b200.so.
//
// Differences a caller may notice:
//  * the class is move-only (the reference's implicit copy double-frees);
//  * fetch samples come in ascending (x, y, z) global-index order (the
//    reference's order is that of its atomics, i.e. unspecified);
//  * update() blocks until the scan is integrated, as the reference's does,
//    unless setAsync(true): then it only enqueues, and any call that reads
//    the map waits for it.
#pragma once

#if __has_include(<Eigen/Dense>)
#include <Eigen/Dense>
#else
#include <cublox/eigen_compat.hpp>
#endif

#include <cublox_b200.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace cublox {

using PointCloud = Eigen::Matrix<float, Eigen::Dynamic, 3>;

// Probability -> log-odds, clamped to [1e-6, 1 - 1e-6] (utils.hpp:185-188).
inline float logit(const float p) {
  const float pc = std::clamp(p, 1.0e-6f, 1.0f - 1.0e-6f);
  return std::log(pc / (1.0f - pc));
}

namespace detail {
inline void ok(int rc, const char *what) {
  if (rc != CUBLOX_OK)
    throw std::runtime_error(std::string("cublox::") + what + ": " + cublox_last_error());
}
// posToGlobalIndex as the reference computes it on the host (utils.hpp:24-31).
inline int posToGlobalIndex(float pos, float inv, bool ctr) {
  if (ctr) {
    const float s = pos < 0.0f ? -1.0f : 1.0f;
    return static_cast<int>(pos * inv + s * 0.5f);
  }
  return static_cast<int>(std::floor(pos * inv));
}
}  // namespace detail

// Window geometry (Grid.hpp:22-57).
class Grid {
 public:
  struct Config {
    float resolution{0.0f};
    float resolution_inv{0.0f};
    Eigen::Vector3i map_size_i{Eigen::Vector3i::Zero()};
    Eigen::Vector3i half_map_size_i{Eigen::Vector3i::Zero()};
    int voxel_num{0};
    bool origin_at_center{false};
    std::optional<float> recenter_threshold{std::nullopt};
    float recenter_threshold_squared{0.0f};
  } config_;

  Eigen::Vector3f origin_f_, bound_min_f_, bound_max_f_;
  Eigen::Vector3i origin_i_, bound_min_i_, bound_max_i_;

  virtual ~Grid() = default;
  virtual void reset() = 0;
  virtual void resetVoxel(const int hash_id) = 0;

  bool inside(const Eigen::Vector3f &pos) const {
    const Eigen::Vector3i id(
        detail::posToGlobalIndex(pos.x(), config_.resolution_inv, config_.origin_at_center),
        detail::posToGlobalIndex(pos.y(), config_.resolution_inv, config_.origin_at_center),
        detail::posToGlobalIndex(pos.z(), config_.resolution_inv, config_.origin_at_center));
    return inside(id);
  }
  bool inside(const Eigen::Vector3i &id_g) const {
    for (int a = 0; a < 3; ++a)
      if (std::abs(id_g(a) - origin_i_(a)) > config_.half_map_size_i(a)) return false;
    return true;
  }
  Eigen::Vector3i getOriginIndex() const { return origin_i_; }
  Eigen::Vector3f getOriginPosition() const { return origin_f_; }

  // Horizontal (xy) margin to the window edge in metres (Grid.cpp:67-78).
  float maxHorizontalInWindowRadius(const Eigen::Vector3f &center) const {
    const int cx = detail::posToGlobalIndex(center.x(), config_.resolution_inv,
                                            config_.origin_at_center);
    const int cy = detail::posToGlobalIndex(center.y(), config_.resolution_inv,
                                            config_.origin_at_center);
    const int mx = config_.half_map_size_i.x() - std::abs(cx - origin_i_.x());
    const int my = config_.half_map_size_i.y() - std::abs(cy - origin_i_.y());
    if (mx < 0 || my < 0) return 0.0f;
    return static_cast<float>(std::min(mx, my)) * config_.resolution;
  }

 protected:
  void setBounds(const Eigen::Vector3i &o) {
    origin_i_ = o;
    const auto pos = [this](int g) {
      return config_.origin_at_center ? g * config_.resolution
                                      : (g + 0.5f) * config_.resolution;
    };
    origin_f_ = Eigen::Vector3f(pos(o.x()), pos(o.y()), pos(o.z()));
    bound_max_i_ = o + config_.half_map_size_i;
    bound_min_i_ = o - config_.half_map_size_i;
    bound_min_f_ = Eigen::Vector3f(pos(bound_min_i_.x()), pos(bound_min_i_.y()),
                                   pos(bound_min_i_.z()));
    bound_max_f_ = Eigen::Vector3f(pos(bound_max_i_.x()), pos(bound_max_i_.y()),
                                   pos(bound_max_i_.z()));
  }
};

class OccupancyGrid : public Grid {
 public:
  enum class VoxelState { UNKNOWN = 0, FREE = 1, OCCUPIED = 2 };
  struct OccupancySample {
    Eigen::Vector3f position;
    VoxelState state;
  };

  OccupancyGrid(const Eigen::Vector3i &half_map_size_i, const float resolution,
                const bool origin_at_center, const std::optional<double> recenter_threshold,
                const Eigen::Vector3f &origin = Eigen::Vector3f::Zero()) {
    const int half[3] = {half_map_size_i.x(), half_map_size_i.y(), half_map_size_i.z()};
    const float o[3] = {origin.x(), origin.y(), origin.z()};
    detail::ok(cublox_grid_create(half, resolution, origin_at_center ? 1 : 0,
                                  recenter_threshold.has_value() ? 1 : 0,
                                  recenter_threshold.value_or(0.0), o, nullptr, &g_),
               "Grid");
    int map[3], hf[3], vn = 0, ctr = 0;
    float res = 0.0f;
    detail::ok(cublox_grid_geometry(g_, map, hf, &vn, &res, &ctr), "Grid");
    config_.resolution = res;
    config_.resolution_inv = 1.0f / res;
    config_.map_size_i = Eigen::Vector3i(map[0], map[1], map[2]);
    config_.half_map_size_i = Eigen::Vector3i(hf[0], hf[1], hf[2]);
    config_.voxel_num = vn;
    config_.origin_at_center = ctr != 0;
    if (recenter_threshold.has_value()) {
      config_.recenter_threshold = static_cast<float>(recenter_threshold.value());
      config_.recenter_threshold_squared =
          config_.recenter_threshold.value() * config_.recenter_threshold.value();
    }
    refreshOrigin();
    std::cout << "cublox::Grid initialized with " << config_.voxel_num << " voxels."
              << std::endl;
  }
  OccupancyGrid() = default;
  ~OccupancyGrid() override { cublox_grid_destroy(g_); }
  OccupancyGrid(const OccupancyGrid &) = delete;
  OccupancyGrid &operator=(const OccupancyGrid &) = delete;
  OccupancyGrid(OccupancyGrid &&o) noexcept : Grid(o) { std::swap(g_, o.g_); async_ = o.async_; }
  OccupancyGrid &operator=(OccupancyGrid &&o) noexcept {
    Grid::operator=(o);
    std::swap(g_, o.g_);
    async_ = o.async_;
    return *this;
  }

  void reset() override {
    if (!g_) return;
    detail::ok(cublox_grid_reset(g_), "reset");
  }
  void resetVoxel(const int hash_id) override {
    if (!g_) return;
    detail::ok(cublox_grid_reset_voxel(g_, hash_id), "resetVoxel");
  }

  // update(cloud, sensor_origin) — world-frame points (OccupancyGrid.cpp:181-238).
  void update(const PointCloud &input_cloud, const Eigen::Vector3f &sensor_origin) {
    if (!g_ || input_cloud.rows() <= 0) return;
    const float so[3] = {sensor_origin.x(), sensor_origin.y(), sensor_origin.z()};
    detail::ok(cublox_grid_update(g_, input_cloud.col(0).data(), input_cloud.col(1).data(),
                                  input_cloud.col(2).data(),
                                  static_cast<int>(input_cloud.rows()), so),
               "update");
    if (!async_) detail::ok(cublox_grid_synchronize(g_), "update");
    refreshOrigin();
  }

  // update() from a sensor-frame cloud and the sensor pose (rotation
  // row-major, translation = sensor origin): the range filter and transform
  // the reference's driver applies before update() (src/main.cpp:640-693),
  // done on the device.  Not in the reference class.
  void updateFromSensor(const PointCloud &cloud_sensor, const float rotation_row_major[9],
                        const Eigen::Vector3f &translation) {
    if (!g_ || cloud_sensor.rows() <= 0) return;
    const float t[3] = {translation.x(), translation.y(), translation.z()};
    detail::ok(cublox_grid_update_pose(g_, cloud_sensor.col(0).data(), CUBLOX_LAYOUT_SOA,
                                       static_cast<int>(cloud_sensor.rows()), rotation_row_major,
                                       t),
               "updateFromSensor");
    if (!async_) detail::ok(cublox_grid_synchronize(g_), "updateFromSensor");
    refreshOrigin();
  }

  // Sliding-window recenter (OccupancyGrid.cpp:141-179).
  void recenter(const Eigen::Vector3f &pos) {
    if (!g_) return;
    const float p[3] = {pos.x(), pos.y(), pos.z()};
    int action = 0;
    detail::ok(cublox_grid_recenter(g_, p, &action), "recenter");
    if (action) refreshOrigin();
  }

  std::vector<OccupancySample> fetchOccupancyAround(
      const Eigen::Vector3f &center, const float radius,
      const std::optional<VoxelState> state_filter = std::nullopt,
      const int max_results = 0) const {
    std::vector<OccupancySample> out;
    if (!g_) return out;
    const float c[3] = {center.x(), center.y(), center.z()};
    const int flt = state_filter ? static_cast<int>(*state_filter) : CUBLOX_FILTER_ALL;
    int64_t n = 0;
    detail::ok(cublox_grid_fetch_counts(g_, c, 1, radius, flt, max_results, &n),
               "fetchOccupancyAround");
    if (n <= 0) return out;
    std::vector<float> pos(3 * static_cast<size_t>(n));
    std::vector<uint8_t> st(static_cast<size_t>(n));
    int64_t got = 0;
    detail::ok(cublox_grid_fetch(g_, c, radius, flt, max_results, pos.data(), st.data(), n, &got),
               "fetchOccupancyAround");
    out.reserve(static_cast<size_t>(got));
    for (int64_t i = 0; i < got; ++i)
      out.push_back({Eigen::Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                     static_cast<VoxelState>(st[i])});
    return out;
  }

  inline void setMaxRaycastRange(const float range) {
    if (g_) detail::ok(cublox_grid_set_max_range(g_, range), "setMaxRaycastRange");
  }
  inline float getMaxRaycastRange() const {
    float r = 25.0f;
    if (g_) detail::ok(cublox_grid_get_max_range(g_, &r), "getMaxRaycastRange");
    return r;
  }
  void setLogOddsParams(const float l_hit, const float l_miss, const float l_min,
                        const float l_max, const float l_free, const float l_occupied) {
    l_free_ = l_free;
    l_occupied_ = l_occupied;
    if (g_)
      detail::ok(cublox_grid_set_log_odds(g_, l_hit, l_miss, l_min, l_max, l_free, l_occupied),
                 "setLogOddsParams");
  }
  inline float getResolutionInv() const { return config_.resolution_inv; }
  inline bool getOriginAtCenter() const { return config_.origin_at_center; }

  bool isOccupied(const Eigen::Vector3f &pos) const { return stateAt(pos) == VoxelState::OCCUPIED; }
  bool isUnknown(const Eigen::Vector3f &pos) const { return stateAt(pos) == VoxelState::UNKNOWN; }
  bool isFree(const Eigen::Vector3f &pos) const { return stateAt(pos) == VoxelState::FREE; }
  bool isOccupied(const Eigen::Vector3i &id_g) const {
    return inside(id_g) && classify(storedAt(hashOf(id_g))) == VoxelState::OCCUPIED;
  }
  bool isUnknown(const Eigen::Vector3i &id_g) const {
    return !inside(id_g) || classify(storedAt(hashOf(id_g))) == VoxelState::UNKNOWN;
  }
  bool isFree(const Eigen::Vector3i &id_g) const {
    return inside(id_g) && classify(storedAt(hashOf(id_g))) == VoxelState::FREE;
  }
  bool isOccupied(const int hash_id) const { return classify(storedAt(hash_id)) == VoxelState::OCCUPIED; }
  bool isUnknown(const int hash_id) const { return classify(storedAt(hash_id)) == VoxelState::UNKNOWN; }
  bool isFree(const int hash_id) const { return classify(storedAt(hash_id)) == VoxelState::FREE; }

  // Many point queries in one launch (isOccupied/isFree/isUnknown by state).
  std::vector<VoxelState> queryStates(const std::vector<Eigen::Vector3f> &pts) const {
    std::vector<float> xyz(3 * pts.size());
    for (size_t i = 0; i < pts.size(); ++i)
      for (int a = 0; a < 3; ++a) xyz[3 * i + a] = pts[i](a);
    std::vector<uint8_t> st(pts.size());
    detail::ok(cublox_grid_query_states(g_, xyz.data(), static_cast<int>(pts.size()), st.data()),
               "queryStates");
    std::vector<VoxelState> out(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) out[i] = static_cast<VoxelState>(st[i]);
    return out;
  }

  void setAsync(bool on) { async_ = on; }
  cublox_grid *handle() const { return g_; }

 private:
  cublox_grid *g_ = nullptr;
  bool async_ = false;
  float l_free_ = -0.0004f, l_occupied_ = 1.7346f;  // OccupancyGrid.hpp:166-167

  void refreshOrigin() {
    int o[3];
    float of[3];
    detail::ok(cublox_grid_origin(g_, o, of), "origin");
    setBounds(Eigen::Vector3i(o[0], o[1], o[2]));
  }
  VoxelState classify(float stored) const {
    if (stored >= l_occupied_) return VoxelState::OCCUPIED;
    if (stored < l_free_) return VoxelState::FREE;
    return VoxelState::UNKNOWN;
  }
  float storedAt(int hash_id) const {
    float v = 0.0f;
    detail::ok(cublox_grid_stored_at(g_, hash_id, &v), "storedAt");
    return v;
  }
  int hashOf(const Eigen::Vector3i &id_g) const {
    int l[3];
    for (int a = 0; a < 3; ++a) {
      const int m = config_.map_size_i(a), h = config_.half_map_size_i(a);
      int v = id_g(a) % m;
      if (v > h) v -= m;
      else if (v < -h) v += m;
      l[a] = v + h;
    }
    return l[0] * config_.map_size_i.y() * config_.map_size_i.z() +
           l[1] * config_.map_size_i.z() + l[2];
  }
  VoxelState stateAt(const Eigen::Vector3f &pos) const {
    if (!inside(pos)) return VoxelState::UNKNOWN;
    const Eigen::Vector3i id(
        detail::posToGlobalIndex(pos.x(), config_.resolution_inv, config_.origin_at_center),
        detail::posToGlobalIndex(pos.y(), config_.resolution_inv, config_.origin_at_center),
        detail::posToGlobalIndex(pos.z(), config_.resolution_inv, config_.origin_at_center));
    return classify(storedAt(hashOf(id)));
  }
};

}  // namespace cublox
