"""FP64 restatement of CTL's geometry encoding for the simple systems it ships:
a cylindrical or flat-panel detector on a tubular or C-arm gantry, driven by
one of the stock trajectory protocols.  Test infrastructure only: it checks
the device encoder (ctlcu_encode_geometry); nothing in the product imports it.

Every step cites the reference file (modules/src/...) and line it follows:

  encodeFullGeometry          acquisition/geometryencoder.cpp:67-81 (prepareView per view)
  encodeSingleViewGeometry    acquisition/geometryencoder.cpp:85-117
  finalSourcePosition         acquisition/geometryencoder.cpp:227-231 (focal spot at 0)
  intrinsicParameterMatrix    acquisition/geometryencoder.cpp:262-290
  ProjectionMatrix::compose   mat/projectionmatrix.cpp:31-48;  normalize :125-131
  rotationMatrix(angle, axis) mat/matrix_utils.tpp:21-41
  TubularGantry               components/tubulargantry.cpp:53-90
  CarmGantry                  components/carmgantry.cpp:34-71
  AbstractGantry composition  components/abstractgantry.h:159-244 (no displacements)
  CylindricalDetector         components/cylindricaldetector.cpp:84-140, :270-283
  FlatPanelDetector           components/flatpaneldetector.cpp:47-50, :84-88
  Helical/Wobble/CirclePlusLine/ShortScan/AxialScan protocols
                              acquisition/trajectories.cpp:30-273

Pinned against the reference's own golden geometries testing/testData/tubeGeo.den
and cArmGeo.den, whose inputs are the ones of testing/src/geometrytest.cpp:17-55
(tests/test_geometry.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PI = math.pi
PI_2 = math.pi / 2.0


def rotation(angle: float, axis: str) -> np.ndarray:
    """mat::rotationMatrix(angle, Qt::Axis) (matrix_utils.tpp:21-41)."""
    s, c = math.sin(angle), math.cos(angle)
    if axis == "x":
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]], dtype=np.float64)
    if axis == "y":
        return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], dtype=np.float64)
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]], dtype=np.float64)


@dataclass
class Detector:
    """CylindricalDetector(nbPixelPerModule, pixelDimensions, nbModules,
    angulationPerModule, moduleSpacing); flat panel: one module, no angulation."""
    channels: int
    rows: int
    pixel_w: float
    pixel_h: float
    modules: int = 1
    angulation: float = 0.0
    spacing: float = 0.0
    skew: float = 0.0
    flat_panel: bool = False

    def module_width(self) -> float:  # cylindricaldetector.cpp:280-283
        return float(self.channels) * self.pixel_w

    def curvature_radius(self) -> float:  # cylindricaldetector.cpp:84-93
        if abs(self.angulation) <= 1e-12:  # qFuzzyIsNull: flat, infinite radius
            return float(np.finfo(np.float64).max)
        d = self.spacing + self.module_width() * math.cos(self.angulation / 2.0)
        return d / math.sqrt(2.0 * (1.0 - math.cos(self.angulation)))

    def fan_angle(self) -> float:  # cylindricaldetector.cpp:270-274
        return (self.modules - 1) * self.angulation + 2.0 * math.atan(0.5 * self.module_width() /
                                                                      self.curvature_radius())

    def module_locations(self):
        """(position, passive rotation) per module (cylindricaldetector.cpp:104-131;
        flat panel: one module at the origin, flatpaneldetector.cpp:47-50)."""
        if self.flat_panel:
            return [(np.zeros(3), np.eye(3))]
        r = self.curvature_radius()
        pt = np.array([0.0, 0.0, r])
        out = []
        for m in range(self.modules):
            a = (float(m) - float(self.modules) * 0.5 + 0.5) * self.angulation  # :134-140
            R = rotation(a, "y")
            p = R @ pt
            p[2] -= r
            out.append((p, R.T))
        return out


@dataclass
class Trajectory:
    """One of the stock protocols with its gantry (trajectories.cpp)."""
    kind: str                       # helical | axial | wobble | short_scan | circle_plus_line
    # tubular gantry (TubularGantry(SDD, SID, rotation, pitch, tilt))
    sdd: float = 0.0
    sid: float = 0.0
    tilt: float = 0.0
    pitch: float = 0.0              # the gantry's own pitch position (axial scans keep it)
    angle_increment: float = 0.0
    pitch_increment: float = 0.0
    start_pitch: float = 0.0
    start_angle: float = 0.0
    # C-arm gantry (CarmGantry(span)) and its protocols
    carm_span: float = 0.0
    source_to_iso: float = 0.0
    angle_span: float = 0.0
    wobble_angle: float = 0.0
    wobble_freq: float = 0.0
    line_length: float = 0.0
    line_fraction: float = 0.0


def _tubular(rotation_angle, pitch, tilt, sdd, sid):
    """Source position, detector position, detector passive rotation and source
    rotation of a TubularGantry (tubulargantry.cpp:53-90)."""
    G = rotation(tilt, "x") @ rotation(rotation_angle, "z")
    src = G @ np.array([sid, 0.0, -pitch])
    src_rot = G @ rotation(PI_2, "z") @ rotation(-PI_2, "x")
    det = G @ np.array([-(sdd - sid), 0.0, -pitch])
    det_rot = (G @ rotation(PI_2, "z") @ rotation(-PI_2, "x")).T
    return src, det, det_rot, src_rot


def _carm(position, rot, span):
    """CarmGantry with location (position, rot) (carmgantry.cpp:34-71)."""
    det = position - rot @ np.array([0.0, 0.0, -span])
    return position, det, rot.T, rot


def _fixed(start_angle):
    # trajectories.cpp:80-81 (and the same line in the other C-arm protocols)
    return rotation(PI_2 + start_angle, "z") @ rotation(-PI_2, "x")


def gantry_state(t: Trajectory, view: int, n_views: int, det: Detector):
    """The gantry after the protocol's prepare step for `view` (trajectories.cpp)."""
    if t.kind == "helical":  # :30-44
        ang = view * t.angle_increment + t.start_angle
        pitch = view * t.pitch_increment + t.start_pitch
        return _tubular(ang, pitch, t.tilt, t.sdd, t.sid)
    if t.kind == "axial":  # :251-265, the increment is a float there (360 deg / views, rounded)
        inc = np.float32(2.0 * PI / n_views) if n_views > 0 else np.float32(0.0)
        ang = float(np.float32(np.float32(view) * inc)) + t.start_angle
        return _tubular(ang, t.pitch, t.tilt, t.sdd, t.sid)
    src0 = np.array([0.0, 0.0, -t.source_to_iso])
    fixed = _fixed(t.start_angle)
    if t.kind == "wobble":  # :66-88
        inc = t.angle_span / float(n_views - 1) if n_views > 1 else 0.0
        phase = math.sin(float(view) / float(n_views) * 2.0 * PI * t.wobble_freq)
        rot = rotation(view * inc, "z") @ fixed @ rotation(phase * t.wobble_angle, "x")
        return _carm(rot @ src0, rot, t.carm_span)
    if t.kind == "short_scan":  # :170-196, span < 0: 180 deg + fan angle (:205-230)
        span = t.angle_span
        if span < 0.0:
            if det.flat_panel:
                width = det.module_width()
            else:
                width = 2.0 * det.curvature_radius() * math.sin(det.fan_angle() / 2.0)
            # the protocol's fan angle is 2 tan(...) of the half width over the span (:229)
            span = PI + 2.0 * math.tan(0.5 * width / t.carm_span)
        inc = span / float(n_views - 1) if n_views > 1 else 0.0
        rot = rotation(view * inc, "z") @ fixed
        return _carm(rot @ src0, rot, t.carm_span)
    if t.kind == "circle_plus_line":  # :114-153
        n_line = int(math.floor(n_views * t.line_fraction))
        n_circle = n_views - n_line
        if view < n_circle:
            inc = t.angle_span / float(n_circle - 1) if n_circle > 1 else 0.0
            rot = rotation(view * inc, "z") @ fixed
            pos = rot @ src0
        else:
            lv = view - n_circle
            linc = t.line_length / float(n_line - 1) if n_line > 1 else 0.0
            rot = rotation(t.angle_span / 2.0, "z") @ fixed
            pos = rot @ src0
            pos[2] += (lv - n_line / 2.0) * linc
        return _carm(pos, rot, t.carm_span)
    raise ValueError(t.kind)


def intrinsic(dev, det: Detector) -> np.ndarray:
    """intrinsicParameterMatrix (geometryencoder.cpp:262-290)."""
    focal = abs(dev[2])
    fx, fy = focal / det.pixel_w, focal / det.pixel_h
    dx = dev[0] / det.pixel_w
    dy = dev[1] / det.pixel_h
    dx += dy * det.skew / fy
    px = 0.5 * float(det.channels - 1) - dx
    py = 0.5 * float(det.rows - 1) - dy
    return np.array([[fx, det.skew, px], [0.0, fy, py], [0.0, 0.0, 1.0]])


def encode_full_geometry(det: Detector, traj: Trajectory, n_views: int, source_shift=None) -> np.ndarray:
    """(n_views, modules, 3, 4) normalised projection matrices
    (geometryencoder.cpp:67-117, projectionmatrix.cpp:44-48, :125-131).
    source_shift: a source displacement (x, y, z) in the source frame, added to
    the prepared gantry as a GantryDisplacementParam increment does
    (preparesteps.cpp:202-210; abstractgantry.h:159-164)."""
    locs = det.module_locations()
    out = np.zeros((n_views, len(locs), 3, 4))
    for v in range(n_views):
        src, det_pos, det_rot, src_rot = gantry_state(traj, v, n_views, det)
        if source_shift is not None:
            src = src + src_rot @ np.asarray(source_shift, np.float64)
        for m, (p, R) in enumerate(locs):
            mod_pos = det_pos + det_rot.T @ p
            tot = R @ det_rot
            K = intrinsic(tot @ (mod_pos - src), det)
            M = K @ tot
            P = np.concatenate([M, (-M @ src)[:, None]], axis=1)
            den = math.copysign(np.linalg.norm(M[2]), np.linalg.det(M))
            out[v, m] = P / den
    return out


def pmat_difference(a: np.ndarray, b: np.ndarray) -> float:
    """Mean Frobenius norm of the difference of the normalised matrices
    (the measure of testing/src/geometrytest.cpp:122-139)."""
    def norm(P):
        M = P[..., :3]
        den = np.linalg.norm(M[..., 2, :], axis=-1) * np.sign(np.linalg.det(M))
        return P / den[..., None, None]
    d = norm(np.asarray(a, np.float64)) - norm(np.asarray(b, np.float64))
    return float(np.sqrt((d ** 2).sum(axis=(-1, -2))).mean())


def golden_tube_setup():
    """geometrytest.cpp:21-25, :42-44: CylindricalDetector(QSize(16, 64), QSizeF(1, 1), 40,
    1 deg, 0.2), TubularGantry(1000, 550, 0, 90 deg, 0 deg), HelicalTrajectory(3.6 deg, 1.0), 10 views."""
    det = Detector(16, 64, 1.0, 1.0, modules=40, angulation=math.radians(1.0), spacing=0.2)
    traj = Trajectory("helical", sdd=1000.0, sid=550.0, tilt=0.0, pitch=math.radians(90.0),
                      angle_increment=math.radians(3.6), pitch_increment=1.0)
    return det, traj, 10


def golden_carm_setup():
    """geometrytest.cpp:21-25, :50-52: the same detector, CarmGantry(1200),
    WobbleTrajectory(200 deg, 750, 0 deg, 20 deg, 5.0), 30 views."""
    det = Detector(16, 64, 1.0, 1.0, modules=40, angulation=math.radians(1.0), spacing=0.2)
    traj = Trajectory("wobble", carm_span=1200.0, source_to_iso=750.0, angle_span=math.radians(200.0),
                      start_angle=0.0, wobble_angle=math.radians(20.0), wobble_freq=5.0)
    return det, traj, 30


def focal_spot_grid(nx: int, ny: int):
    """ArealFocalSpotExtension::discretizationGrid (arealfocalspotextension.cpp):
    nx x ny points in [-1/2, 1/2]^2, x outer, y inner (one point: the centre)."""
    xs = [-0.5 + i / (nx - 1) for i in range(nx)] if nx > 1 else [0.0]
    ys = [-0.5 + j / (ny - 1) for j in range(ny)] if ny > 1 else [0.0]
    return [(x, y) for x in xs for y in ys]
