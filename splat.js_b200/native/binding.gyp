# node-gyp build of the Node-API addon over libsplat_b200.so:
#   cd splat.js_b200/native && node-gyp rebuild
# (build the library first: python splat.js_b200/build.py)
{
  "targets": [
    {
      "target_name": "gs_b200",
      "sources": ["gs_b200_napi.c"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/..", "-lsplat_b200", "-Wl,-rpath,<(module_root_dir)/.."],
      "cflags": ["-std=c11", "-Wall", "-Wextra"],
      "defines": ["_POSIX_C_SOURCE=200809L"]
    }
  ]
}
