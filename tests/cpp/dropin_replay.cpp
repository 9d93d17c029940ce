// The C++ drop-in (include/cublox/OccupancyGrid.hpp) driven as the
// reference's own C++ callers drive theirs, linked with libcublox_b200.so.
//
//   dropin_replay replay IN OUT
//       Reads a scenario written by tests/test_cpp_dropin.py: grid arguments,
//       log-odds, max range, a scan and its sensor origin, a recenter
//       position, fetch centres and radius, query points.  Constructs a
//       cublox::OccupancyGrid, calls update, recenter, fetchOccupancyAround
//       (all states and OCCUPIED-only, capped and not), isOccupied / isFree /
//       isUnknown by position, global index and hash, inside,
//       maxHorizontalInWindowRadius, getMaxRaycastRange, resetVoxel and
//       reset, and writes every answer to OUT for the test to compare with
//       the oracle.
//
//   dropin_replay perf [N_ITERS]
//       The reference's own perf test restated (test/test_occupancy_grid_perf
//       .cpp:31-100): a 401 x 401 x 201 grid at 0.05 m, origin at the
//       centre, no recenter threshold; 500,000 points on a [1.5, 8] m
//       spherical shell around the sensor at the origin (std::mt19937 seed
//       42, radius, cos(theta) and phi uniform); one warm-up update, then
//       N_ITERS timed updates (default 100); prints the same lines.
#include <cublox/OccupancyGrid.hpp>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <vector>

namespace {

struct Reader {
  FILE *f;
  template <class T>
  T get() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) throw std::runtime_error("short input");
    return v;
  }
  template <class T>
  std::vector<T> vec(size_t n) {
    std::vector<T> v(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) throw std::runtime_error("short input");
    return v;
  }
};

struct Writer {
  FILE *f;
  template <class T>
  void put(const T &v) {
    std::fwrite(&v, sizeof(T), 1, f);
  }
  template <class T>
  void put_vec(const std::vector<T> &v) {
    put<int64_t>(static_cast<int64_t>(v.size()));
    if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
  }
};

using VS = cublox::OccupancyGrid::VoxelState;

void put_origin(Writer &w, const cublox::OccupancyGrid &g) {
  const Eigen::Vector3i o = g.getOriginIndex();
  const Eigen::Vector3f of = g.getOriginPosition();
  for (int a = 0; a < 3; ++a) w.put<int32_t>(o(a));
  for (int a = 0; a < 3; ++a) w.put<float>(of(a));
}

void put_fetch(Writer &w, const std::vector<cublox::OccupancyGrid::OccupancySample> &s) {
  std::vector<float> pos;
  std::vector<uint8_t> st;
  for (const auto &x : s) {
    for (int a = 0; a < 3; ++a) pos.push_back(x.position(a));
    st.push_back(static_cast<uint8_t>(x.state));
  }
  w.put_vec(pos);
  w.put_vec(st);
}

uint8_t state_bits(bool occ, bool fre, bool unk) {
  return static_cast<uint8_t>((occ ? 2 : (fre ? 1 : 0)) | (unk ? 4 : 0));
}

int replay(const char *in_path, const char *out_path) {
  FILE *fi = std::fopen(in_path, "rb");
  FILE *fo = std::fopen(out_path, "wb");
  if (!fi || !fo) {
    std::fprintf(stderr, "cannot open input or output\n");
    return 2;
  }
  Reader r{fi};
  Writer w{fo};
  const int hx = r.get<int32_t>(), hy = r.get<int32_t>(), hz = r.get<int32_t>();
  const float res = r.get<float>();
  const int ctr = r.get<int32_t>();
  const double thr = r.get<double>();
  const float max_range = r.get<float>();
  const auto lo = r.vec<float>(6);
  const int64_t n = r.get<int64_t>();
  const auto pts = r.vec<float>(3 * static_cast<size_t>(n));
  const auto sensor = r.vec<float>(3);
  const auto rc_pos = r.vec<float>(3);
  const int64_t nc = r.get<int64_t>();
  const auto centres = r.vec<float>(3 * static_cast<size_t>(nc));
  const float radius = r.get<float>();
  const int64_t nq = r.get<int64_t>();
  const auto queries = r.vec<float>(3 * static_cast<size_t>(nq));
  std::fclose(fi);

  cublox::OccupancyGrid g(Eigen::Vector3i(hx, hy, hz), res, ctr != 0,
                          thr > 0.0 ? std::optional<double>(thr) : std::nullopt);
  g.setLogOddsParams(lo[0], lo[1], lo[2], lo[3], lo[4], lo[5]);
  g.setMaxRaycastRange(max_range);
  w.put<float>(g.getMaxRaycastRange());
  w.put<int32_t>(g.config_.voxel_num);
  put_origin(w, g);

  cublox::PointCloud cloud(n, 3);
  for (int64_t i = 0; i < n; ++i)
    for (int a = 0; a < 3; ++a) cloud(i, a) = pts[3 * i + a];
  const Eigen::Vector3f so(sensor[0], sensor[1], sensor[2]);
  g.update(cloud, so);
  put_origin(w, g);  // the first update snaps the window to the sensor
  g.recenter(Eigen::Vector3f(rc_pos[0], rc_pos[1], rc_pos[2]));
  put_origin(w, g);

  for (int64_t c = 0; c < nc; ++c) {
    const Eigen::Vector3f ce(centres[3 * c], centres[3 * c + 1], centres[3 * c + 2]);
    put_fetch(w, g.fetchOccupancyAround(ce, radius));
    put_fetch(w, g.fetchOccupancyAround(ce, radius, VS::OCCUPIED));
    put_fetch(w, g.fetchOccupancyAround(ce, radius, std::nullopt, 7));
    w.put<float>(g.maxHorizontalInWindowRadius(ce));
  }
  // point queries by position and by global index; every voxel of a slab
  // through the window's centre by hash
  std::vector<uint8_t> by_pos, by_idx, inside, by_hash;
  const auto &cfg = g.config_;
  for (int64_t q = 0; q < nq; ++q) {
    const Eigen::Vector3f p(queries[3 * q], queries[3 * q + 1], queries[3 * q + 2]);
    by_pos.push_back(state_bits(g.isOccupied(p), g.isFree(p), g.isUnknown(p)));
    inside.push_back(g.inside(p) ? 1 : 0);
    Eigen::Vector3i id;
    for (int a = 0; a < 3; ++a)
      id(a) = cublox::detail::posToGlobalIndex(p(a), cfg.resolution_inv, cfg.origin_at_center);
    by_idx.push_back(state_bits(g.isOccupied(id), g.isFree(id), g.isUnknown(id)));
  }
  const int ny = cfg.map_size_i.y(), nz = cfg.map_size_i.z();
  const int sx = cfg.half_map_size_i.x();
  for (int sy = 0; sy < ny; ++sy)
    for (int sz = 0; sz < nz; ++sz) {
      const int h = (sx * ny + sy) * nz + sz;
      by_hash.push_back(state_bits(g.isOccupied(h), g.isFree(h), false));
    }
  w.put_vec(by_pos);
  w.put_vec(by_idx);
  w.put_vec(inside);
  w.put_vec(by_hash);
  // resetVoxel of the first occupied voxel on the slab, then reset()
  int first = -1;
  for (size_t k = 0; k < by_hash.size() && first < 0; ++k)
    if (by_hash[k] == 2) first = (sx * ny) * nz + static_cast<int>(k);
  w.put<int32_t>(first);
  if (first >= 0) {
    g.resetVoxel(first);
    w.put<uint8_t>(g.isUnknown(first) ? 1 : 0);
  }
  g.reset();
  int64_t left = 0;
  for (int64_t c = 0; c < nc; ++c) {
    const Eigen::Vector3f ce(centres[3 * c], centres[3 * c + 1], centres[3 * c + 2]);
    for (const auto &s : g.fetchOccupancyAround(ce, radius))
      if (s.state != VS::UNKNOWN) ++left;
  }
  w.put<int64_t>(left);
  std::fclose(fo);
  return 0;
}

cublox::PointCloud shell_cloud(int n, float r_min, float r_max, std::uint32_t seed) {
  cublox::PointCloud cloud(n, 3);
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> r_dist(r_min, r_max);
  std::uniform_real_distribution<float> u_dist(-1.0f, 1.0f);
  std::uniform_real_distribution<float> phi_dist(0.0f, 2.0f * static_cast<float>(M_PI));
  for (int i = 0; i < n; ++i) {
    const float rr = r_dist(rng);
    const float ct = u_dist(rng);
    const float st = std::sqrt(std::max(0.0f, 1.0f - ct * ct));
    const float phi = phi_dist(rng);
    cloud(i, 0) = rr * st * std::cos(phi);
    cloud(i, 1) = rr * st * std::sin(phi);
    cloud(i, 2) = rr * ct;
  }
  return cloud;
}

int perf(int iters) {
  cublox::OccupancyGrid grid(Eigen::Vector3i(200, 200, 100), 0.05f, true, std::nullopt,
                             Eigen::Vector3f::Zero());
  constexpr int kNumPoints = 500000;
  const auto cloud = shell_cloud(kNumPoints, 1.5f, 8.0f, 42);
  const Eigen::Vector3f sensor = Eigen::Vector3f::Zero();
  auto bench_one = [&]() {
    const auto t0 = std::chrono::steady_clock::now();
    grid.update(cloud, sensor);
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
  };
  std::printf("grid: %d x %d x %d voxels (%d total) at %.2f m resolution\n",
              grid.config_.map_size_i.x(), grid.config_.map_size_i.y(),
              grid.config_.map_size_i.z(), grid.config_.voxel_num,
              static_cast<double>(grid.config_.resolution));
  std::printf("cloud: %d points on a [%.1f, %.1f] m spherical shell\n", kNumPoints, 1.5, 8.0);
  std::printf("warm-up update():     %.3f ms\n", bench_one());
  double total = 0.0, mn = std::numeric_limits<double>::max(), mx = 0.0;
  for (int i = 0; i < iters; ++i) {
    const double ms = bench_one();
    total += ms;
    mn = std::min(mn, ms);
    mx = std::max(mx, ms);
  }
  const double mean = total / iters;
  std::printf("steady-state over %d iters: mean=%.3f ms, min=%.3f ms, max=%.3f ms  (~%.1f Hz "
              "at mean)\n",
              iters, mean, mn, mx, 1000.0 / mean);
  // the shell's voxels are occupied after so many hits
  const auto s = grid.fetchOccupancyAround(Eigen::Vector3f(4.0f, 0.0f, 0.0f), 0.5f,
                                           cublox::OccupancyGrid::VoxelState::OCCUPIED);
  std::printf("occupied samples within 0.5 m of (4, 0, 0): %zu\n", s.size());
  return s.empty() ? 1 : 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    if (argc >= 4 && std::strcmp(argv[1], "replay") == 0) return replay(argv[2], argv[3]);
    if (argc >= 2 && std::strcmp(argv[1], "perf") == 0)
      return perf(argc >= 3 ? std::atoi(argv[2]) : 100);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
  std::fprintf(stderr, "usage: dropin_replay replay IN OUT | perf [N]\n");
  return 2;
}
