"""Import shim for ``astropy.io.fits``; any call raises."""


def open(*args, **kwargs):  # noqa: A001
    raise NotImplementedError("astropy.io.fits stand-in: inject arrays instead")


def getdata(*args, **kwargs):
    raise NotImplementedError("astropy.io.fits stand-in: inject arrays instead")
