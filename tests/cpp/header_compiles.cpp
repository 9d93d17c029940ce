// Compile-only check of the C++ drop-in header over the C ABI, with the
// Eigen stand-in (no Eigen on this machine).
#include <cublox/OccupancyGrid.hpp>

int use_api(cublox::OccupancyGrid &g, const cublox::PointCloud &cloud) {
  const float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  g.update(cloud, Eigen::Vector3f(0.0f, 0.0f, 1.8f));
  g.updateFromSensor(cloud, R, Eigen::Vector3f(0.0f, 0.0f, 1.8f));
  g.recenter(Eigen::Vector3f(1.0f, 0.0f, 1.8f));
  auto s = g.fetchOccupancyAround(Eigen::Vector3f(0.0f, 0.0f, 1.0f), 1.0f);
  return static_cast<int>(s.size());
}
