#include "dataset.h"

#include <fstream>
#include <stdexcept>

namespace ursus {
namespace io {

DataSet::DataSet(ui dims, ui n, std::string path, DataSetType set_type, DataType dtype,
                 ClusterType ctype, std::string rebuild)
    : number_of_dimensions(dims), number_of_data(n), data_set_path(path), data_set_type(set_type),
      data_type(dtype), cluster_type(ctype), force_rebuild(rebuild) {
  std::ifstream in(path, std::ios::in | std::ios::binary);
  if (!in) throw std::runtime_error("Failed to open a file(" + path + ")");
  points.resize((size_t)dims * n);
  in.read(reinterpret_cast<char*>(points.data()), (std::streamsize)(sizeof(Point) * points.size()));
  if ((size_t)in.gcount() != sizeof(Point) * points.size())
    throw std::runtime_error("short read from " + path);
}

DataSet::DataSet(ui dims, std::vector<Point> rows)
    : number_of_dimensions(dims), number_of_data((ui)(rows.size() / (dims ? dims : 1))),
      data_set_type(DATASET_TYPE_BINARY), data_type(DATA_TYPE_SYNTHETIC),
      cluster_type(CLUSTER_TYPE_HILBERT), points(std::move(rows)), force_rebuild("no") {}

}  // namespace io
}  // namespace ursus
