"""B200-native (sm_100a) point-source model-map path of xtsrcmaps.

The package holds the host-side mirror of the reference's three namespace
entry points (Exposure::compute_exposure, Psf::compute_psf_data,
ModelMap::compute_srcmaps) over the C-ABI library ``libxts_cuda.so`` built from
``xtsrcmaps_b200/csrc``.
"""
