// Minimal HDF5 files without libhdf5: a root group of contiguous datasets,
// written and read following the HDF5 File Format Specification (version 3.0)
// -- superblock version 2, version-2 object headers with Jenkins lookup3
// checksums, a compact ("new-style") root group of Link messages, and
// datasets with a version-2 dataspace, an IEEE little-endian f64 or i32
// datatype, a version-3 fill value message and a contiguous layout.  This is
// the subset the reference's output files use (mod_hdf5.cc: 3-D f64 datasets
// and 1-element int "attribute" datasets), readable by any HDF5 library
// 1.10 or later.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace plc {
namespace h5 {

enum class Type { F64, I32 };

struct Dataset {
  std::string name;
  Type type = Type::F64;
  std::vector<uint64_t> dims;  // slowest first, as HDF5 stores them
  const void *data = nullptr;  // dims-product elements, little-endian
};

// Jenkins' lookup3 hashlittle (the checksum of HDF5 metadata), initval 0.
uint32_t lookup3(const uint8_t *key, size_t length, uint32_t initval = 0);

// Writes the datasets as the members of the root group; false on I/O error.
bool write_file(const std::string &path, const std::vector<Dataset> &sets, std::string &err);

// Reads dataset `name` of the root group into out (converted to double), its
// dims into dims; false (with a message) if the file is not one this reader
// understands or the dataset is missing.
bool read_dataset(const std::string &path, const std::string &name, std::vector<double> &out,
                  std::vector<uint64_t> &dims, std::string &err);

}  // namespace h5
}  // namespace plc
