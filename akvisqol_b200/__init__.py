"""akvisqol_b200: the ViSQOL hot path as sm_100a CUDA kernels behind the
reference's C ABI (include/visqol.h), with its Python binding mirror in
``akvisqol_b200.native``.
"""
