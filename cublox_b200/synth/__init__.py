"""Seeded synthetic LiDAR scenes, scans and trajectories.

Inputs for the parity tests and the benchmark.  The reference's own input (a
recorded LiDAR bag) is not available, so scans are ray-cast from a seeded
scene: the ground plane z = 0 plus axis-aligned boxes standing on it.

Per-scan recipe (shared by every configuration):
  * beams at evenly spaced elevations, azimuths evenly spaced over 360 deg,
    rotated by the sensor yaw; points ordered azimuth-major (all beams of one
    azimuth, then the next), as a spinning LiDAR reports them;
  * the true hit range gets Gaussian noise N(0, sigma);
  * a return whose noisy range exceeds max_range, or a beam that hits
    nothing, becomes a "no-return" endpoint at 1.5 x max_range along the
    beam, which the reference's clip path integrates as free space only
    (src/kernels.cu:57-67);
  * points are world-frame float32, sensor at the given pose.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libcublox_synth.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the C ray caster next to this file (gcc, no GPU needed)."""
    src = os.path.join(_HERE, "scan_synth.c")
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(src)
    ):
        import subprocess

        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-o", _LIB_PATH, src, "-lm", "-lpthread"]
        )
    return _LIB_PATH


def use_library(path: str) -> None:
    """Cast scans with another build of scan_synth.c (same symbols), e.g. one
    linked into a test harness, instead of libcublox_synth.so.  Call before
    the first scan."""
    global _LIB_PATH, _lib
    if _lib is not None and path != _LIB_PATH:
        raise RuntimeError("synth: the caster library is already loaded")
    _LIB_PATH = path


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.synth_cast.argtypes = [dp, dp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
        lib.synth_cast.restype = ctypes.c_int
        _lib = lib
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class Scene:
    boxes: np.ndarray  # (B, 6) float64: xmin, ymin, zmin, xmax, ymax, zmax
    ground: bool = True


def make_scene(seed: int, n_boxes: int, extent: float, side=(0.3, 3.0), height=None,
               keepout=None) -> Scene:
    """Boxes with centres uniform in +-extent (x, y), base on the ground.

    `side` bounds the x/y/z side lengths (uniform); `height`, if given,
    bounds the z side separately.  `keepout(cx, cy, hx, hy) -> bool` rejects
    boxes (resampled) that would sit on the sensor's path.
    """
    rng = np.random.default_rng(seed)
    boxes = []
    tries = 0
    while len(boxes) < n_boxes and tries < 100 * max(n_boxes, 1):
        tries += 1
        cx, cy = rng.uniform(-extent, extent, size=2)
        sx, sy = rng.uniform(side[0], side[1], size=2)
        sz = rng.uniform(height[0], height[1]) if height else rng.uniform(side[0], side[1])
        if keepout is not None and keepout(cx, cy, sx / 2, sy / 2):
            continue
        boxes.append([cx - sx / 2, cy - sy / 2, 0.0, cx + sx / 2, cy + sy / 2, sz])
    return Scene(np.asarray(boxes, dtype=np.float64).reshape(-1, 6))


@dataclass
class Sensor:
    beams: int
    azimuths: int
    elev_min_deg: float
    elev_max_deg: float
    max_range: float
    sigma: float

    @property
    def n_points(self) -> int:
        return self.beams * self.azimuths

    def directions(self, yaw: float = 0.0) -> np.ndarray:
        el = np.deg2rad(np.linspace(self.elev_min_deg, self.elev_max_deg, self.beams))
        az = yaw + 2.0 * np.pi * np.arange(self.azimuths) / self.azimuths
        ce, se = np.cos(el), np.sin(el)
        ca, sa = np.cos(az), np.sin(az)
        d = np.empty((self.azimuths, self.beams, 3), dtype=np.float64)
        d[..., 0] = ca[:, None] * ce[None, :]
        d[..., 1] = sa[:, None] * ce[None, :]
        d[..., 2] = se[None, :]
        return d.reshape(-1, 3)


def cast(scene: Scene, origin, dirs: np.ndarray, threads: int | None = None) -> np.ndarray:
    lib = _load()
    o = np.ascontiguousarray(np.asarray(origin, dtype=np.float64))
    d = np.ascontiguousarray(dirs, dtype=np.float64)
    b = np.ascontiguousarray(scene.boxes, dtype=np.float64)
    out = np.empty(d.shape[0], dtype=np.float64)
    th = threads or min(8, os.cpu_count() or 1)
    rc = lib.synth_cast(_dp(o), _dp(d), d.shape[0], _dp(b), b.shape[0], int(scene.ground), _dp(out), th)
    if rc != 0:
        raise RuntimeError("synth_cast failed")
    return out


def scan(scene: Scene, sensor: Sensor, origin, yaw: float, seed: int) -> np.ndarray:
    """One scan: (N, 3) float32 world-frame points."""
    dirs = sensor.directions(yaw)
    t = cast(scene, origin, dirs)
    rng = np.random.default_rng(seed)
    r = t + rng.normal(0.0, sensor.sigma, size=t.shape)
    no_ret = ~np.isfinite(t) | (r > sensor.max_range)
    r = np.where(no_ret, 1.5 * sensor.max_range, np.maximum(r, 1e-3))
    pts = np.asarray(origin, dtype=np.float64)[None, :] + r[:, None] * dirs
    return pts.astype(np.float32)


# ---------------------------------------------------------------------------
# Trajectories
# ---------------------------------------------------------------------------
def circle_trajectory(n: int, radius: float, speed: float, rate_hz: float, height: float):
    """Poses (x, y, z, yaw) on a circle about the origin, starting at (R, 0)."""
    dth = speed / rate_hz / radius
    th = dth * np.arange(n)
    x = radius * np.cos(th)
    y = radius * np.sin(th)
    yaw = th + np.pi / 2
    return np.stack([x, y, np.full(n, height), yaw], axis=1)


def line_trajectory(n: int, speed: float, rate_hz: float, height: float, start=(0.0, 0.0),
                    heading: float = 0.0):
    step = speed / rate_hz
    s = step * np.arange(n)
    x = start[0] + s * np.cos(heading)
    y = start[1] + s * np.sin(heading)
    return np.stack([x, y, np.full(n, height), np.full(n, heading)], axis=1)


# ---------------------------------------------------------------------------
# The five workloads (log-odds from the reference's yaml defaults).
# ---------------------------------------------------------------------------
YAML_PROBS = dict(hit=0.9, miss=0.49, min=0.12, max=0.98, free=0.499, occupied=0.85)


@dataclass
class Workload:
    name: str
    half: tuple
    resolution: float
    sensor: Sensor
    scene: Scene
    poses: np.ndarray
    threshold: float | None
    seed: int
    fetch_centres: int = 0
    fetch_radius: float = 0.0
    extra: dict = field(default_factory=dict)

    def scan(self, k: int) -> np.ndarray:
        x, y, z, yaw = self.poses[k]
        return scan(self.scene, self.sensor, (x, y, z), yaw, seed=self.seed * 100003 + k)

    def sensor_origin(self, k: int) -> np.ndarray:
        return np.asarray(self.poses[k][:3], dtype=np.float32)


def _keepout_point(px, py, margin):
    def f(cx, cy, hx, hy):
        return abs(cx - px) < hx + margin and abs(cy - py) < hy + margin
    return f


def _keepout_circle(radius, margin):
    def f(cx, cy, hx, hy):
        r = np.hypot(cx, cy)
        return abs(r - radius) < np.hypot(hx, hy) + margin
    return f


def _keepout_line(y0, margin):
    def f(cx, cy, hx, hy):
        return abs(cy - y0) < hy + margin
    return f


def plain_small(threshold: float | None = 4.0) -> Workload:
    """200x200x40 voxels at 0.1 m, one 16x1024 scan from (0, 0, 1.8)."""
    sensor = Sensor(16, 1024, -15.0, 15.0, 20.0, 0.02)
    scene = make_scene(0, 40, 9.0, keepout=_keepout_point(0.0, 0.0, 1.0))
    poses = np.array([[0.0, 0.0, 1.8, 0.0]])
    return Workload("plain_small_201x201x41", (100, 100, 20), 0.1, sensor, scene, poses,
                    threshold, seed=0, fetch_centres=1000, fetch_radius=1.0,
                    extra=dict(recenter_shift=(37, -12, 3)))


def readme_scale(n_scans: int = 200) -> Workload:
    """701x701x151 voxels (74.2M) at 0.1 m, 64x1024 scans, 50 m, circle R=25 m."""
    sensor = Sensor(64, 1024, -22.5, 22.5, 50.0, 0.02)
    scene = make_scene(1, 400, 60.0, keepout=_keepout_circle(25.0, 1.5))
    poses = circle_trajectory(n_scans, 25.0, 1.5, 10.0, 1.8)
    return Workload("readme_701x701x151_64x1024", (350, 350, 75), 0.1, sensor, scene, poses,
                    4.0, seed=1)


def stress(n_scans: int = 300) -> Workload:
    """1025x1025x257 voxels at 0.05 m, 128x2048 scans, 100 m, 8 m/s line."""
    sensor = Sensor(128, 2048, -22.5, 22.5, 100.0, 0.03)
    scene = make_scene(4, 3000, 150.0, side=(1.0, 12.0), height=(2.0, 20.0),
                       keepout=_keepout_line(0.0, 2.0))
    poses = line_trajectory(n_scans, 8.0, 10.0, 1.8, start=(-120.0, 0.0))
    return Workload("stress_1025x1025x257_128x2048", (512, 512, 128), 0.05, sensor, scene,
                    poses, 0.5, seed=4, fetch_centres=10000, fetch_radius=2.0)


BATCH_DIMS = ((128, 128, 32), (200, 200, 40), (256, 256, 64))  # 257x257x65, 401x401x81, 513x513x129


@dataclass
class BatchWorkload:
    """Many independent maps, one scan per map per step, uneven point counts.

    Map m has grid half-size `halves[m]`, its own box scene and a straight
    line trajectory; at step k its scan has `counts[m, k]` points from a
    `beams`-beam sensor (counts[m, k] / beams azimuths)."""
    name: str
    halves: list
    resolution: float
    beams: int
    elev: tuple
    max_range: float
    sigma: float
    scenes: list
    poses: list
    counts: np.ndarray
    threshold: float | None
    seed: int

    @property
    def n_maps(self) -> int:
        return len(self.halves)

    def sensor(self, m: int, k: int) -> Sensor:
        return Sensor(self.beams, int(self.counts[m, k]) // self.beams, self.elev[0], self.elev[1],
                      self.max_range, self.sigma)

    def sensor_origin(self, m: int, k: int) -> np.ndarray:
        return np.asarray(self.poses[m][k][:3], dtype=np.float32)

    def scan(self, m: int, k: int) -> np.ndarray:
        x, y, z, yaw = self.poses[m][k]
        return scan(self.scenes[m], self.sensor(m, k), (x, y, z), yaw,
                    seed=(self.seed * 1000 + m) * 100003 + k)

    def step(self, k: int):
        """All maps' scans of step k: (list of (N_m, 3) arrays, (n_maps, 3) sensors)."""
        return ([self.scan(m, k) for m in range(self.n_maps)],
                np.stack([self.sensor_origin(m, k) for m in range(self.n_maps)]))


def batching(n_maps: int = 32, n_steps: int = 100, dims=BATCH_DIMS, n_min: int = 8192,
             n_max: int = 131072, beams: int = 32, max_range: float = 30.0, speed: float = 2.0,
             rate_hz: float = 10.0, threshold: float | None = 4.0, n_boxes: int = 200,
             seed: int = 2) -> BatchWorkload:
    """`n_maps` grids drawn from `dims` at 0.1 m, point counts uniform in
    [n_min, n_max] (rounded down to whole azimuth columns), 32-beam sensor
    over +-15 deg, 30 m range, straight lines at 2 m/s, 10 Hz."""
    rng = np.random.default_rng(seed)
    halves = [tuple(dims[i]) for i in rng.integers(0, len(dims), size=n_maps)]
    counts = rng.integers(n_min, n_max + 1, size=(n_maps, n_steps))
    counts = np.maximum(counts // beams, 1) * beams
    scenes, poses = [], []
    for m in range(n_maps):
        y0 = float(rng.uniform(-5.0, 5.0))
        scenes.append(make_scene(seed * 1000 + m, n_boxes, 45.0, keepout=_keepout_line(y0, 1.5)))
        poses.append(line_trajectory(n_steps, speed, rate_hz, 1.8, start=(-10.0, y0)))
    return BatchWorkload(f"batch{n_maps}_" + "|".join(f"{2*a+1}x{2*b+1}x{2*c+1}" for a, b, c in dims),
                         halves, 0.1, beams, (-15.0, 15.0), max_range, 0.02, scenes, poses,
                         counts, threshold, seed)


SERVE_DIMS = ((200, 200, 40), (350, 350, 75))  # 401x401x81, 701x701x151
SERVE_SENSORS = ((16, 1024, 15.0), (64, 1024, 22.5), (128, 2048, 22.5))  # beams, azimuths, +-elev


@dataclass
class ServeWorkload:
    """Requests of many robots arriving over time.

    Robot r has map half-size `halves[r]`, a box scene and a circle
    trajectory; its scans come from `pool[r][c][j]` = (points, sensor
    origin), size class c, pose j, reused cyclically along the trajectory.
    `events` is a time-ordered list of (t_seconds, kind, robot, c, j) with
    kind "scan" or "fetch" (c, j unused for fetches; `fetch_centres(i)`
    gives the i-th fetch's centres)."""
    name: str
    halves: list
    resolution: float
    max_range: float
    threshold: float | None
    pool: list
    events: list
    fetch_n: int
    fetch_radius: float
    seed: int

    @property
    def n_robots(self) -> int:
        return len(self.halves)

    def fetch_centres(self, i: int, robot: int, origin) -> np.ndarray:
        rng = np.random.default_rng((self.seed * 7919 + i) & 0xffffffff)
        c = np.empty((self.fetch_n, 3), dtype=np.float32)
        c[:, 0] = origin[0] + rng.uniform(-10.0, 10.0, self.fetch_n)
        c[:, 1] = origin[1] + rng.uniform(-10.0, 10.0, self.fetch_n)
        c[:, 2] = rng.uniform(0.0, 3.0, self.fetch_n)
        return c


def serving(n_robots: int = 16, seconds: float = 60.0, scan_rate: float = 400.0,
            fetch_rate: float = 100.0, dims=SERVE_DIMS, sensors=SERVE_SENSORS,
            probs=(0.5, 0.35, 0.15), poses: int = 6, max_range: float = 50.0,
            threshold: float | None = 4.0, fetch_n: int = 256, fetch_radius: float = 1.5,
            n_boxes: int = 200, seed: int = 3) -> ServeWorkload:
    """Poisson arrivals of scans (aggregate `scan_rate`/s, point counts by
    `sensors` with probabilities `probs`) and fetches (`fetch_rate`/s, each
    `fetch_n` centres around the robot), robots picked uniformly."""
    rng = np.random.default_rng(seed)
    halves = [tuple(dims[i]) for i in rng.integers(0, len(dims), size=n_robots)]
    pool = []
    for r in range(n_robots):
        scene = make_scene(seed * 1000 + r, n_boxes, 60.0, keepout=_keepout_circle(15.0, 1.5))
        traj = circle_trajectory(poses, 15.0, 1.5, 10.0, 1.8)
        classes = []
        for c, (beams, az, el) in enumerate(sensors):
            sen = Sensor(beams, az, -el, el, max_range, 0.02)
            classes.append([(scan(scene, sen, tuple(traj[j][:3]), traj[j][3],
                                  seed=(seed * 100 + r) * 1009 + c * 101 + j),
                             np.asarray(traj[j][:3], dtype=np.float32)) for j in range(poses)])
        pool.append(classes)
    events = []
    for kind, rate in (("scan", scan_rate), ("fetch", fetch_rate)):
        t = 0.0
        while True:
            t += rng.exponential(1.0 / rate)
            if t >= seconds:
                break
            events.append((t, kind, int(rng.integers(0, n_robots)),
                           int(rng.choice(len(sensors), p=probs)), 0))
    events.sort(key=lambda e: e[0])
    count = [0] * n_robots
    out = []
    for t, kind, r, c, _ in events:
        if kind == "scan":
            out.append((t, kind, r, c, count[r] % poses))
            count[r] += 1
        else:
            out.append((t, kind, r, 0, 0))
    return ServeWorkload(f"serve{n_robots}_" + "|".join(f"{2*a+1}x{2*b+1}x{2*c+1}" for a, b, c in dims),
                         halves, 0.1, max_range, threshold, pool, out, fetch_n, fetch_radius, seed)


def perf_test_cloud(n: int = 500000, r_min: float = 1.5, r_max: float = 8.0, seed: int = 42):
    """Spherical-shell cloud with the shape of the reference's perf test
    (test/test_occupancy_grid_perf.cpp:31-50): radius uniform in
    [r_min, r_max], direction uniform on the sphere, about the origin."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(r_min, r_max, n)
    ct = rng.uniform(-1.0, 1.0, n)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    return np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], axis=1).astype(np.float32)
