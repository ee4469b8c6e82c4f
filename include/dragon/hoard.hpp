// DRAGONHOARD over the C ABI: output and restart from device buffers
// (DRAGONHOARD/DragonHoard.hpp:16-33, DRAGONHOARD_Config.h:16-35).
//
// The reference's compile-time switches are run-time settings here
// (DRAGONHOARD::options); the file layout, keys and flattening are the
// reference's (HDF5_Attrs.hpp:14-59, HDF5Output.cpp:308), written by the
// library's own HDF5 writer, so no HDF5 installation is needed.
#pragma once

#include <string>

#include "dragon.hpp"

namespace DRAGONHOARD {

inline std::string output_base_name = "frame";  // files are <output_base_name>_#####.h5
inline std::string output_dir = "";
inline int restart_frame = 0;  // RESTART_FRAME: < 0 restarts from the highest-numbered file

struct Options {
    int write_option = 3;       // HDF5_WRITE_OPTION: 1 primitive, 3 + energy, 6 conservative, 7 both
    int redundant_vals = 1;     // HDF5_REDUNDANT_VALS_OPTION: 0 omit, 1 float, 2 double
    int compression_level = 4;  // HDF5_COMPRESSION_LEVEL: <= 0 writes contiguous, uncompressed datasets
    bool write_ghosts = false;  // WRITE_GHOSTS_TO_FILE
    int threads = 0;            // host threads that deflate chunks; 0: every core
};
inline Options options;

// writeToFile (HDF5Output.cpp:103-528): output_dir + "/" + filename + ".h5",
// complete when the call returns.
void writeToFile(dragon::Grid& grid, double t, int cycle, const std::string& filename);
// The same snapshot, taken now and written while the caller keeps stepping;
// waitForFiles returns once every file of the grid is complete.
void writeToFileAsync(dragon::Grid& grid, double t, int cycle, const std::string& filename);
void waitForFiles(dragon::Grid& grid);
// loadFromFile (HDF5Restart.cpp:61-377): restarts the grid from
// output_dir + "/" + filename (".h5" appended when missing); the grid's
// spacing becomes the file's. Throws std::runtime_error with the reference's
// messages on a dimension, size or physics mismatch.
void loadFromFile(dragon::Grid& grid, double& t, int& cycle, const std::string& filename);
void verifyOutputDirectory();   // OutputDir.cpp:18-27
std::string restartFileName();  // OutputDir.cpp:29-72
std::string cycle_string(int n);

}  // namespace DRAGONHOARD
