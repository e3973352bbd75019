{
  "targets": [
    {
      "target_name": "efs_napi",
      "sources": ["efs_napi.cc"],
      "include_dirs": ["../include"],
      "libraries": ["-L<(module_root_dir)/../efs_b200", "-lefs", "-Wl,-rpath,<(module_root_dir)/../efs_b200"],
      "cflags_cc": ["-std=c++17", "-O2"]
    }
  ]
}
