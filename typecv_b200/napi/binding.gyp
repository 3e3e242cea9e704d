# node-gyp build of the N-API addon over libtba.so (unbuilt here: no Node toolchain in this image).
#   python -m typecv_b200.build   # typecv_b200/libtba.so for sm_100a
#   node-gyp rebuild              # from this directory
{
  "targets": [{
    "target_name": "tba_napi",
    "sources": ["tba_napi.c"],
    "include_dirs": ["../../include"],
    "libraries": ["-L<(module_root_dir)/..", "-ltba", "-Wl,-rpath,<(module_root_dir)/.."],
    "cflags": ["-std=c11", "-O2", "-Wall"]
  }]
}
