// One configuration file run the way the reference's `bubbles` program runs
// it (src/bubbles.cpp:190-310): parse, the transducer.pid_iterate passes,
// rawdata, focal-point tracker files, *_minmax.txt and runtime.txt.  Shared by
// `bubbles` and `bubbles_series`.
#pragma once
#include <ostream>
#include <string>

struct ConfRun {
  std::string in_file;
  std::string target_dir = "./rawdata/";
  bool ascii = false;      // -a
  bool sph = false;        // -s
  bool dir_given = false;  // -d given: pid_iterate passes write to <dir>_I/, <dir>_II/, ...
  bool progress = true;    // the reference's progress line on stdout at each save
  bool banner = true;      // "Input file is ..." lines
};

// Returns the program's exit status (0, or 1 after printing the error to err).
int run_configuration(const ConfRun& run, std::ostream& out, std::ostream& err);
