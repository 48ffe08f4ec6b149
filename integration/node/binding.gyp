{
  # node-gyp build of the `fdtd_b200` N-API module (binding_b200.cpp) for
  # js_fdtd/src/backends/b200/.  The CUDA code is not compiled here: the module
  # links the prebuilt libfdtd_b200.so (python -c "import __graft_entry__ as g;
  # g.build()" at the root of this repository builds it for sm_100a).
  # Set B200_ROOT to that repository root:
  #   B200_ROOT=/path/to/repo node-gyp configure build
  "variables": {
    "b200_root%": "<!(node -e \"process.stdout.write(process.env.B200_ROOT || '')\")"
  },
  "targets": [
    {
      "target_name": "fdtd_b200",
      "sources": ["binding_b200.cpp"],
      "include_dirs": [
        "<!@(node -p \"require('node-addon-api').include\")",
        "<(b200_root)/include"
      ],
      "defines": ["NAPI_VERSION=8", "NAPI_CPP_EXCEPTIONS"],
      "cflags_cc!": ["-fno-exceptions"],
      "cflags_cc": ["-std=c++17", "-fexceptions"],
      "libraries": [
        "-L<(b200_root)/special-topics_b200/_build",
        "-lfdtd_b200",
        "-Wl,-rpath,<(b200_root)/special-topics_b200/_build"
      ]
    }
  ]
}
