"""crystal-b200: B200-native execution layer for crystal-sycl's fused star-join
query pipeline (fact scan -> predicate -> dimension perfect-hash build/probe ->
group-by aggregate).

The product is libcrystal_b200.so (include/crystal_b200.h): NVRTC-compiled
sm_100a kernels generated from star-join plans, run by a generic executor.  This
package binds it (``_lib``), builds plans (``plan``, ``queries``), generates
synthetic SSB-shaped tables (``datagen``) and keeps tables resident on the GPU
(``engine``).  Importing ``practice_b200._lib`` (which every module that runs
queries does) loads the library and raises if it is missing; the package
itself imports nothing so that ``python -m practice_b200.build`` can build it.
"""
