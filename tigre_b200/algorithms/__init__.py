"""Device-resident algorithm drivers with the reference's names and signatures
(Python/tigre/algorithms/__init__.py): fdk/FDK, fbp, cgls, lsqr, lsmr, ossart, sirt, sart, sart_tv, ossart_tv, mlem, fista, ista and
the POCS family (asd_pocs, awasd_pocs, os_asd_pocs, os_awasd_pocs, piccs, os_piccs, pcsd, aw_pcsd,
os_pcsd, os_aw_pcsd)."""
from .krylov import (cgls, cgls_device, lsqr, lsmr, hybrid_lsqr, ab_gmres, ba_gmres, irn_tv_cgls,  # noqa: F401
                     hybrid_flsqr_tv)
from .single_pass import FDK, fdk, fbp, fdk_device  # noqa: F401
from .art import ossart, sirt, sart, sart_tv, ossart_tv, ART  # noqa: F401
from .statistical import mlem  # noqa: F401
from .pocs import (asd_pocs, awasd_pocs, os_asd_pocs, os_awasd_pocs, piccs, os_piccs, pcsd, aw_pcsd,  # noqa: F401
                   os_pcsd, os_aw_pcsd)
from .ista import fista, ista  # noqa: F401

__all__ = ["FDK", "fdk", "fbp", "cgls", "lsqr", "lsmr", "ossart", "sirt", "sart", "asd_pocs", "fista", "ista", "awasd_pocs",
           "os_asd_pocs", "os_awasd_pocs", "piccs", "os_piccs", "pcsd", "aw_pcsd", "os_pcsd", "os_aw_pcsd",
           "sart_tv", "ossart_tv", "mlem",
           "hybrid_lsqr", "ab_gmres", "ba_gmres", "irn_tv_cgls", "hybrid_flsqr_tv"]
