"""Import-only stand-in for the absent netCDF4 package: the reference's
forcing modules import it at module level, but the functions the golden
generator calls (the seasonal blend) never open a file.  Any use raises."""


class Dataset:  # noqa: D101
    def __init__(self, *args, **kwargs):
        raise RuntimeError("netCDF4 is not available; the golden generator does not read NetCDF files")
