"""B200-native EAM force-and-stress path for mdelast: the CUDA library and the pybind11
module md_driver_module (built into mdelast_b200/lib by mdelast_b200.build), and the host
side around them (potential files, lattices and cells, the elastic-constant protocol, the
learned warm start, the statistical benchmarks)."""
