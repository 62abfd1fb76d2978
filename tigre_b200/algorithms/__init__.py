"""Device-resident algorithm drivers with the reference's names and signatures
(Python/tigre/algorithms/__init__.py): fdk/FDK, fbp, cgls, lsqr, lsmr, ossart, sirt, sart, asd_pocs, fista, ista."""
from .krylov import cgls, cgls_device, lsqr, lsmr  # noqa: F401
from .single_pass import FDK, fdk, fbp, fdk_device  # noqa: F401
from .art import ossart, sirt, sart, ART  # noqa: F401
from .pocs import asd_pocs  # noqa: F401
from .ista import fista, ista  # noqa: F401

__all__ = ["FDK", "fdk", "fbp", "cgls", "lsqr", "lsmr", "ossart", "sirt", "sart", "asd_pocs", "fista", "ista"]
