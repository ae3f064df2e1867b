"""Drop-in for the reference package `pydiffbmp` (smhongok/diffbmp) on the
rasterizer's path: SimpleTileRenderer's render, batch render and fit loop,
and DiffBMPWrapper's render / render_batch, computed by libdbmp.so's sm_100a
kernels.  A caller that puts diffbmp_b200/ on sys.path imports it as
`pydiffbmp`.  The reference's asset loaders, initializers, exporters and CLI
are not part of this path."""
