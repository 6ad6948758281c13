"""CPU restatement of SnapshotManager::SaveFrame's record logic
(simulation/snapshotmanager.cpp:160-262, converter/visualpoint.h:7-21) in
float32 numpy arithmetic without fused multiply-adds, as the reference's host
Eigen code computes it. Test infrastructure: only tests/ use it, as the
checker of mpm_frame_records.

State kept between frames (snapshotmanager.h:30-31): visual_state (float
pos, vel, Jp_inv, status byte) and last_pos_refresh_frame. The partial-frame
loop reads `VisualPoint vp = visual_state[count]` by value (:177), so its
refreshed values never reach visual_state; only last_pos_refresh_frame
changes.
"""
import numpy as np

from icempm_3dm_b200.layout import IDX_JP_INV, IDX_UTILITY, POSX, VELX

STATUS_CRUSHED, STATUS_DISABLED = 0x10000, 0x20000
THRESHOLD_JP = np.float32(1e-2)


def _points(soa):
    u = soa[IDX_UTILITY].view(np.int64)
    keep = (u & STATUS_DISABLED) == 0
    pos = soa[POSX:POSX + 3, keep].astype(np.float32)
    vel = soa[VELX:VELX + 3, keep].astype(np.float32)
    jp = soa[IDX_JP_INV, keep].astype(np.float32)
    uk = u[keep]
    status = (((uk >> 24) & 0xFF) | np.where(uk & STATUS_CRUSHED, 0x80, 0)).astype(np.uint8)
    return pos, vel, jp, status


class FrameState:
    def __init__(self):
        self.pos = self.vel = self.jp = self.status = self.last = None

    def full(self, soa, frame):
        """:166-187: the VisualPoint records; keeps them as the visual state."""
        pos, vel, jp, status = _points(soa)
        self.pos, self.vel, self.jp, self.status = pos, vel, jp, status
        self.last = np.full(pos.shape[1], frame, dtype=np.int64)
        return pos, vel, jp, status

    def partial(self, soa, frame, dt, coeff, threshold_pos):
        """:199-238: (pos/vel index, Jp index, status index) arrays of the
        points with UpdatePos, UpdateJp and UpdateStatus records, in order,
        plus the current float values (pos, vel, jp, status)."""
        pos, vel, jp, status = _points(soa)
        elapsed = frame - self.last
        f = (dt * elapsed.astype(np.float64) * float(coeff)).astype(np.float32)
        with np.errstate(over="ignore", invalid="ignore"):
            pred = self.pos + self.vel * f[None, :]          # float32 products, then sums
            e = pos - pred
            n2 = (e[0] * e[0] + e[1] * e[1]) + e[2] * e[2]
        upd_pv = np.sqrt(n2).astype(np.float64) > threshold_pos
        self.last[upd_pv] = frame
        upd_jp = np.abs(self.jp - jp) > THRESHOLD_JP
        upd_st = self.status != status
        return (np.flatnonzero(upd_pv), np.flatnonzero(upd_jp), np.flatnonzero(upd_st)), (pos, vel, jp, status)
