{
  "targets": [
    {
      "target_name": "courant_napi",
      "sources": ["courant_napi.cc", "shim.cpp", "shim_exports.cpp", "arena.cpp"],
      "cflags_cc": ["-std=c++17", "-O2", "-fexceptions"],
      "cflags_cc!": ["-fno-exceptions"],
      "libraries": ["-ldl"]
    }
  ]
}
