// A small HDF5 writer and reader for the solver's snapshot files, written for this project from
// the public HDF5 File Format Specification (no libhdf5 in this build).
//
// Writer: the layout libhdf5 produces with its default (earliest-format) properties, which every
// HDF5 reader opens:
//   - superblock version 0, 8-byte offsets and lengths, group leaf/internal node K = 4/16;
//   - the root group as an "old-style" symbol-table group: a version-1 B-tree node of type 0, one
//     symbol table node (SNOD) and a local heap holding the link names;
//   - version-1 object headers;
//   - datasets: simple dataspaces (version 1), IEEE little-endian 64-bit floats, contiguous
//     storage (layout message version 3), a fill-value message (version 2, no fill value);
//   - attributes of the root group: scalar 64-bit floats or 32-bit signed integers (attribute
//     message version 1).
// At most 8 datasets (one symbol table node); names shorter than 256 bytes.
//
// Reader: superblock versions 0 to 3; symbol-table groups (any B-tree depth) and compact
// link-message groups; object header versions 1 and 2 with continuation blocks; dataspace
// versions 1 and 2; layout versions 3 and 4 (contiguous and compact storage); attribute message
// versions 1 to 3; IEEE floats of 4 or 8 bytes and integers of 1 to 8 bytes of either byte order.
// Datasets or attributes in other forms (chunked or compressed storage, dense attribute or link
// storage, shared messages, variable-length types) are rejected with an error naming them.
#pragma once
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

namespace h5lite {

struct WriteDataset {
    std::string name;
    std::vector<uint64_t> dims;   // row-major, the last dimension fastest
    const double* data;           // prod(dims) values
};

struct WriteAttr {
    std::string name;
    bool is_int = false;
    double d = 0.0;
    int32_t i = 0;
};

// Writes a new file (replacing any old one). Returns false with a message in err.
bool write_file(const std::string& path, const std::vector<WriteDataset>& datasets,
                const std::vector<WriteAttr>& root_attrs, std::string& err);

class File {
  public:
    File() = default;
    ~File();
    File(const File&) = delete;
    File& operator=(const File&) = delete;
    bool open(const std::string& path, std::string& err);
    // links of the root group and their object header addresses
    const std::map<std::string, uint64_t>& links() const { return links_; }
    bool has(const std::string& name) const { return links_.count(name) != 0; }
    // a scalar numeric attribute of the root group, converted to double; false when absent
    bool attr(const std::string& name, double& v) const;
    // a numeric dataset of the root group, converted to double
    bool read(const std::string& name, std::vector<uint64_t>& dims, std::vector<double>& out, std::string& err);

  private:
    struct Msg {
        uint16_t type;
        uint8_t flags;
        std::vector<uint8_t> data;
    };
    struct Type {
        int cls = -1;       // 0 fixed-point, 1 floating point
        int size = 0;
        bool big_endian = false, is_signed = false;
    };
    bool read_at(uint64_t addr, void* dst, size_t n) const;
    uint64_t get_uint(const uint8_t* p, int n) const;
    bool object_header(uint64_t addr, std::vector<Msg>& out, std::string& err) const;
    bool read_symbol_table(uint64_t btree, uint64_t heap, std::string& err);
    bool btree_node(uint64_t addr, uint64_t heap_data, int depth, std::string& err);
    bool decode_type(const uint8_t* p, size_t n, Type& t) const;
    bool convert(const uint8_t* src, const Type& t, uint64_t count, double* dst) const;
    FILE* f_ = nullptr;
    uint64_t base_ = 0, eof_ = 0;
    int so_ = 8, sl_ = 8;            // sizes of offsets and lengths
    std::map<std::string, uint64_t> links_;
    std::map<std::string, double> attrs_;
};

}  // namespace h5lite
