"""Drop-in ``core`` package: the hot-path modules of AstroFD's core/ package
(srhd_core, rmhd_core, boundary, nozzle, source_terms) backed by
libastrofd_b200.so."""
