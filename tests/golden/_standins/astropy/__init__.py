"""Import shim: the reference imports ``astropy.io.fits`` at module level only
for file-based map I/O, which the golden-vector runs never use (arrays are
injected through the in-memory seams)."""
