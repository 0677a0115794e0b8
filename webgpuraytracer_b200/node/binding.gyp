{
  "targets": [
    {
      "target_name": "wgpt",
      "sources": ["addon.cc"],
      "include_dirs": ["../../include"],
      "cflags_cc": ["-std=c++17", "-fexceptions"],
      "cflags_cc!": ["-fno-exceptions"],
      "libraries": ["-L<(module_root_dir)/../_lib", "-lwgpt", "-Wl,-rpath,<(module_root_dir)/../_lib"]
    }
  ]
}
