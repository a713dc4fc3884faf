"""Reading forcepho's image stores and packing patches from them.

* ``fits``    -- FITS headers, images and binary tables (read and write)
* ``wcs``     -- TAN (gnomonic) world coordinate systems, ``scale_at_sky``
* ``h5lite``  -- HDF5 groups, attributes and datasets (superblock v0)
* ``region``  -- ``CircularRegion``, ``RectangularRegion``
* ``patch``   -- ``FITSPatch``, ``StorePatch``, ``PSFStore``, ``PixelStore``, ``MetaStore``
"""
