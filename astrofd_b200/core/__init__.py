"""Drop-in ``core`` package: the hot-path modules of AstroFD's core/ package
(srhd_core, rmhd_core, boundary, nozzle, source_terms, chemistry,
dissipation, and the fixed-metric wrappers grhd_core, grmhd_core, gr_metric)
backed by libastrofd_b200.so."""
