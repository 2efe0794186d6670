"""B200 (sm_100a) implementation of the OpenIFS prognostic cloud scheme CLOUDSC.

The product is the C-ABI library ``libcloudsc_b200.so`` (include/cloudsc_b200.h);
this package builds it (``openifs_b200.build``), binds it (``openifs_b200.cloudsc``)
and generates seeded synthetic inputs (``openifs_b200.inputs``).
"""
from .params import CloudscParams  # noqa: F401
