"""``healpy.rotator.Rotator`` stand-in: ZYZ Euler (0, 90, 0) only (test-only)."""
import numpy as np

from oracle.dsht_oracle import rotate_points, rotate_alm_back


class Rotator:
    def __init__(self, rot=None, coord=None, inv=False, deg=True, eulertype="ZYX"):
        rot = tuple(float(r) for r in (rot if rot is not None else (0, 0, 0)))
        if eulertype != "ZYZ" or not deg or rot != (0.0, 90.0, 0.0):
            raise NotImplementedError("only Rotator(rot=(0,90,0), eulertype='ZYZ', deg=True)")
        self.inv = bool(inv)

    def __call__(self, theta, phi):
        return rotate_points(theta, phi, inverse=self.inv)

    def rotate_alm(self, alm, lmax=None, mmax=None, inplace=False):
        if not self.inv:
            raise NotImplementedError("only the inverse rotation of alm is used by the reference")
        alm = np.asarray(alm, dtype=np.complex128)
        Nl = int(round((np.sqrt(8 * alm.size + 1) - 1) / 2))
        return rotate_alm_back(alm, Nl)
