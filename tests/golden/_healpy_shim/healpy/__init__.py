"""Test-only stand-in for the parts of healpy that the reference's ``sht/sht.py``
touches (``import healpy as hp`` at :9 and ``hp.rotator.Rotator`` at :134-139).

healpy is not installed in this environment.  The rotation it stands in for is the
oracle's restatement (``oracle.dsht_oracle.rotate_points`` / ``rotate_alm_back``).
Used only by ``tests/golden/make_golden.py`` to import and run the reference.
"""
from . import rotator  # noqa: F401
