"""SnapshotManager of the reference (simulation/snapshotmanager.{h,cpp}) on
the HDF5 codec of h5io: the raw point-cloud loader, the full snapshot
d%05d.h5 (checkpoint) and resume from it, the animation frames v%05d.h5,
plus the parameter attributes of SimParams3D (parameters_sim_3d.cpp:178-282).

The files carry the reference's dataset names, shapes, element types,
chunking, deflate levels and attribute names and types, in the reference's
order. The host SoA is the reference's HostSideSOA buffer: 28 rows
of `capacity` doubles (row k at offset k * capacity), `size` of them in use.

RemoveDisabledAndSort, which LoadRawPoints and ReadSnapshot run on the host
in the reference, runs on the device here (mpm_sort, the same stable
cell-key order) when the model uploads the points.
"""
import math
import os
import time

import numpy as np

from ._lib import FE00, IDX_JP_INV, IDX_UTILITY, LIB, N_PTS_ARRAYS, POSX, STATUS_LIQUID, SimParams3D
from .h5io import H5File, H5Writer

I32, U32, U8, U64, F64 = np.int32, np.uint32, np.uint8, np.uint64, np.float64

# SimParams3D::SaveParametersAsAttributes, in its order (parameters_sim_3d.cpp:178-282)
PARAM_ATTRS = (
    ("SetupType", I32),
    ("nPtsTotal", I32), ("GridXTotal", I32), ("GridY", I32), ("GridZ", I32), ("cellsize", F64),
    ("IndenterSubdivisions", I32),
    ("InitialTimeStep", F64), ("SimulationEndTime", F64), ("SimulationTime", F64), ("UpdateEveryNthStep", I32),
    ("SnapshotPeriod", I32), ("SimulationStep", I32),
    ("Gravity", F64), ("Density", F64), ("PoissonsRatio", F64), ("YoungsModulus", F64),
    ("IceCompressiveStrength", F64), ("IceTensileStrength", F64), ("IceTensileStrength2", F64),
    ("IceShearStrength", F64), ("DP_tan_phi", F64), ("DP_threshold_p", F64), ("GrainVariability", F64),
    ("indenter_x", F64), ("indenter_y", F64), ("indenter_x_initial", F64), ("indenter_y_initial", F64),
    ("IndDiameter", F64), ("IndVelocity", F64),
    ("ParticleVolume", F64), ("ParticleMass", F64), ("Volume", F64),
    ("nPartitions", I32), ("GridHaloSize", I32), ("PointTransferFrequency", I32),
    ("ExtraSpaceForIncomingPoints", F64), ("PointsTransferBufferFraction", F64),
    ("RebalanceThresholdFreeSpaceRemaining", F64), ("RebalanceThresholdDisabledPercentage", F64),
    ("animation_threshold_pos", F64),
)

# ReadParametersFromAttributes (parameters_sim_3d.cpp:285-391) opens
# DP_threshold_p but never reads it, so a resumed run has the Reset() value;
# animation_threshold_pos is read only when present.
_NOT_READ = ("DP_threshold_p",)
_OPTIONAL = ("animation_threshold_pos",)


def params_as_attributes(prms):
    """{name: typed scalar} in SaveParametersAsAttributes order."""
    return {name: t(getattr(prms, name)) for name, t in PARAM_ATTRS}


def params_from_attributes(attrs):
    """SimParams3D::ReadParametersFromAttributes: Reset(), the saved values,
    DomainDimensionX = GridXTotal * cellsize, then ComputeCamClayParams and
    ComputeHelperVariables. A missing required attribute raises KeyError."""
    p = SimParams3D()
    LIB.mpm_params_reset(p)
    for name, t in PARAM_ATTRS:
        if name in _NOT_READ:
            continue
        if name not in attrs:
            if name in _OPTIONAL:
                continue
            raise KeyError(f"attribute {name} missing")
        setattr(p, name, t(attrs[name]).item())
    p.DomainDimensionX = p.GridXTotal * p.cellsize
    LIB.mpm_params_compute_camclay(p)
    LIB.mpm_params_compute_helper_variables(p)
    return p


def animation_frame_number(prms):
    """SimParams3D::AnimationFrameNumber (parameters_sim_3d.h:104)."""
    return prms.SimulationStep // prms.UpdateEveryNthStep


def load_raw_points(path, prms):
    """SnapshotManager::LoadRawPoints (snapshotmanager.cpp:20-113) up to the
    upload. Reads llGrainIDs (into the utility row, as raw uint64), x, y, z
    and the 'volume' attribute; places the block as the reference does (x and
    z shifted by (grid length - block length) / 2, y so that the lowest
    point is 2h above the floor; SetupType 2 marks the points outside the
    cutout centred in x and z at the block's top as liquid before the shift); sets
    F = I, Jp_inv = 1 (HostSideSOA::InitializeBlock), the indenter start and
    ParticleVolume = Volume / n. Returns (prms, soa, capacity): a copy of
    prms, the (28, n) SoA in file order (the cell-key sort follows on the
    device), and the host capacity n * (1 + ExtraSpaceForIncomingPoints)."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"error reading raw points file - no file: {path}")
    p = prms.copy() if hasattr(prms, "copy") else prms
    with H5File(path) as f:
        grains = f.read("llGrainIDs").astype(np.uint64)
        n = grains.size
        soa = np.zeros((N_PTS_ARRAYS, n), dtype=np.float64)
        soa[IDX_UTILITY] = grains.view(np.float64)
        for d, k in enumerate("xyz"):
            soa[POSX + d] = f.read(k)
        volume = float(f.attrs("llGrainIDs")["volume"])
    p.nPtsTotal = n
    capacity = int(n * (1 + p.ExtraSpaceForIncomingPoints))
    p.Volume = volume
    pos = soa[POSX:POSX + 3]
    lo, hi = pos.min(axis=1), pos.max(axis=1)
    p.xmin, p.ymin, p.zmin = (float(v) for v in lo)
    p.xmax, p.ymax, p.zmax = (float(v) for v in hi)
    h = p.cellsize
    box_x, box_z = p.GridXTotal * h, p.GridZ * h
    length, width = p.xmax - p.xmin, p.zmax - p.zmin
    x_offset = (box_x - length) / 2
    y_offset = 2 * h - p.ymin
    z_offset = (box_z - width) / 2
    if p.SetupType == 2:
        cut = np.array([p.BlockCutout[0], p.BlockCutout[1], p.BlockCutout[2]])
        centre = (lo + hi) * 0.5
        centre[1] = hi[1] - cut[1] / 2
        a, b = centre - 0.5 * cut, centre + 0.5 * cut
        outside = np.any((pos < a[:, None]) | (pos > b[:, None]), axis=0)
        bits = soa[IDX_UTILITY].view(np.int64)
        bits[outside] |= STATUS_LIQUID
    pos[0] += x_offset
    pos[1] += y_offset
    pos[2] += z_offset
    soa[IDX_JP_INV] = 1.0
    for i in range(3):
        soa[FE00 + 4 * i] = 1.0
    block_left = x_offset
    block_top = p.ymax + y_offset
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    x_ind_offset = math.sqrt(r * r - ht * ht)
    p.indenter_x = math.floor((block_left - x_ind_offset) / h) * h
    if p.SetupType == 0:
        p.indenter_y = block_top + ht
    elif p.SetupType == 1:
        p.indenter_y = math.ceil(block_top / h) * h
    p.indenter_x_initial = p.indenter_x
    p.indenter_y_initial = p.indenter_y
    p.ParticleVolume = p.Volume / n
    LIB.mpm_params_compute_helper_variables(p)
    return p, soa, capacity


def snapshot_path(output_directory, frame):
    return os.path.join(output_directory, f"d{frame:05d}.h5")


def save_snapshot(output_directory, frame, prms, hssoa, size, indenter_sensor_total, compress=False):
    """SnapshotManager::SaveSnapshot (snapshotmanager.cpp:299-340): writes
    d<frame>.h5 with 'Indenter' (3 * IndenterSubdivisions * GridZ doubles)
    and 'Points' (the whole host buffer, capacity * 28 doubles, row k of the
    SoA at k * capacity; chunks of min(2^20, size) elements, deflate 5 when
    compress), with HSSOA_capacity, HSSOA_size (unsigned) and the parameter
    attributes on 'Points'. hssoa is (28, capacity). Returns the path."""
    os.makedirs(output_directory, exist_ok=True)
    hssoa = np.ascontiguousarray(hssoa, dtype=np.float64)
    if hssoa.shape[0] != N_PTS_ARRAYS or size > hssoa.shape[1]:
        raise ValueError("hssoa must be (28, capacity) with size <= capacity")
    capacity = hssoa.shape[1]
    ind = np.ascontiguousarray(indenter_sensor_total, dtype=np.float64).reshape(-1)
    expected = 3 * prms.IndenterSubdivisions * prms.GridZ
    if ind.size != expected:
        raise ValueError(f"indenter sensor array has {ind.size} values, expected {expected}")
    path = snapshot_path(output_directory, frame)
    attrs = {"HSSOA_capacity": U32(capacity), "HSSOA_size": U32(size)}
    attrs.update(params_as_attributes(prms))
    with H5Writer(path) as w:
        w.create_dataset("Indenter", ind)
        kw = {}
        if compress:
            kw = {"chunks": (min(1024 * 1024, int(size)) or 1,), "deflate": 5}
        w.create_dataset("Points", hssoa.reshape(-1), attrs=attrs, **kw)
    return path


def read_snapshot(path, partitions=0):
    """SnapshotManager::ReadSnapshot (snapshotmanager.cpp:346-405) up to the
    upload: returns (prms, hssoa (28, capacity), size, indenter_sensor_total).
    partitions > 0 overrides nPartitions (then ComputeHelperVariables)."""
    if not os.path.exists(path):
        raise FileNotFoundError("snapshot file does not exist")
    with H5File(path) as f:
        attrs = f.attrs("Points")
        p = params_from_attributes(attrs)
        if partitions > 0:
            p.nPartitions = partitions
            LIB.mpm_params_compute_helper_variables(p)
        capacity, size = int(attrs["HSSOA_capacity"]), int(attrs["HSSOA_size"])
        pts = f.read("Points")
        if pts.size != capacity * N_PTS_ARRAYS:
            raise ValueError("Points does not hold capacity * 28 values")
        ind = f.read("Indenter")
    return p, pts.reshape(N_PTS_ARRAYS, capacity), size, ind


# Record types of the animation frames (converter/visualpoint.cpp:12-41),
# with the reference's member names, offsets and sizes.
VISUAL_POINT = np.dtype({"names": ["px", "py", "pz", "vx", "vy", "vz", "Jp_inv", "status"],
                         "formats": ["<f4"] * 7 + ["u1"], "offsets": [0, 4, 8, 12, 16, 20, 24, 28], "itemsize": 32})
UPDATE_POS = np.dtype({"names": ["idx", "px", "py", "pz", "vx", "vy", "vz"], "formats": ["<i4"] + ["<f4"] * 6,
                       "offsets": [0, 4, 8, 12, 16, 20, 24], "itemsize": 28})
UPDATE_JP = np.dtype({"names": ["idx", "Jp_inv"], "formats": ["<i4", "<f4"], "offsets": [0, 4], "itemsize": 8})
UPDATE_STATUS = np.dtype({"names": ["idx", "status"], "formats": ["<i4", "u1"], "offsets": [0, 4], "itemsize": 8})


def frame_path(output_directory, frame):
    return os.path.join(output_directory, f"v{frame:05d}.h5")


def save_frame(output_directory, frame, prms, indenter_sensor_total, indenter_force, previous_frame_exists,
               points=None, upd_pos=None, upd_jp=None, upd_status=None, timestamp=None):
    """SnapshotManager::SaveFrame's file (snapshotmanager.cpp:116-293):
    v<frame>.h5 with 'Indenter' (chunks of min(10000, size), deflate 5) and
    its attributes indenter_total_x/y/z, partial_frame (uint8), the parameter
    attributes and timestamp (uint64, seconds since the epoch); then either
    'VisualPoints' (a full frame, when no previous frame exists; chunks of
    min(2^20, count)) or the non-empty ones of 'UpdatePos', 'UpdateStatus',
    'UpdateJp' (chunks of min(65536, count)), all deflate 5. The records are
    those of mpm_frame_records. Returns the path."""
    os.makedirs(output_directory, exist_ok=True)
    ind = np.ascontiguousarray(indenter_sensor_total, dtype=np.float64).reshape(-1)
    if ind.size != 3 * prms.IndenterSubdivisions * prms.GridZ:
        raise ValueError("indenter sensor array does not match the parameters")
    f = np.asarray(indenter_force, dtype=np.float64).reshape(3)
    attrs = {"indenter_total_x": F64(f[0]), "indenter_total_y": F64(f[1]), "indenter_total_z": F64(f[2]),
             "partial_frame": U8(1 if previous_frame_exists else 0)}
    attrs.update(params_as_attributes(prms))
    attrs["timestamp"] = U64(int(time.time()) if timestamp is None else timestamp)
    path = frame_path(output_directory, frame)
    with H5Writer(path) as w:
        w.create_dataset("Indenter", ind, chunks=(min(10000, ind.size),), deflate=5, attrs=attrs)
        if not previous_frame_exists:
            pts = np.asarray(points, dtype=VISUAL_POINT)
            w.create_dataset("VisualPoints", pts, chunks=(max(1, min(1024 * 1024, pts.size)),), deflate=5)
        else:
            for name, recs, dt in (("UpdatePos", upd_pos, UPDATE_POS), ("UpdateStatus", upd_status, UPDATE_STATUS),
                                   ("UpdateJp", upd_jp, UPDATE_JP)):
                recs = np.asarray(recs, dtype=dt)
                if recs.size:
                    w.create_dataset(name, recs, chunks=(min(1024 * 64, recs.size),), deflate=5)
    return path


def read_frame(path):
    """The contents of a v<frame>.h5 file: {'attrs': Indenter's attributes,
    'Indenter': array, and whichever of 'VisualPoints', 'UpdatePos',
    'UpdateStatus', 'UpdateJp' it holds}."""
    with H5File(path) as f:
        out = {"attrs": f.attrs("Indenter")}
        for k in f.keys():
            out[k] = f.read(k)
    return out
