{
  "targets": [
    {
      "target_name": "shaderous_b200",
      "sources": ["shaderous_addon.cc"],
      "include_dirs": ["<!(node -p \"require('node-addon-api').include_dir\")", "../../include"],
      "defines": ["NAPI_CPP_EXCEPTIONS", "NAPI_VERSION=8"],
      "cflags_cc": ["-std=c++17", "-fexceptions"],
      "libraries": ["-L<(module_root_dir)/..", "-lshaderous_b200", "-Wl,-rpath,<(module_root_dir)/.."]
    }
  ]
}
