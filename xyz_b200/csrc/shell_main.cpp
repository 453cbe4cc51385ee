// xyzgpu_shell: the reference renderer's program (xyz/main.cpp:27-63) on the
// GPU path tracer.  `xyzgpu_shell NAME` runs the script ./NAME.ren; with no
// argument, or when that script cannot be opened, the shell reads commands
// from standard input (the reference opens its preview window there and
// reaches the same shell with the 'x' key).  Commands: include/xyzgpu_shell.hpp.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>

#include "xyzgpu_shell.hpp"

int main(int argc, char **argv) {
  std::fprintf(stderr, "XYZGPU (build %s, %s)\n", __DATE__, __TIME__);
  xyzgpu::Shell::Config cfg;
  cfg.program = xyzgpu::shell_detail::PathToName(argv[0]);
  xyzgpu::Shell shell(cfg);
  if (argc > 1) {
    std::ifstream fin(cfg.ren_dir + argv[1] + ".ren");
    if (fin) return shell.Run(fin, false);
  }
  return shell.Run(std::cin, true);
}
