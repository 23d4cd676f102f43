{
  "targets": [{
    "target_name": "lvbh_napi",
    "sources": ["lvbh_napi.cc"],
    "include_dirs": ["../../include"],
    "libraries": ["-L<(module_root_dir)/../lvbh", "-llvbh", "-Wl,-rpath,<(module_root_dir)/../lvbh"],
    "cflags_cc": ["-std=c++17"]
  }]
}
