// Index persistence in the reference's file layout (reference:
// nsparse/io/index_io.h:20-36, io/io.h). Files written here load in the
// reference and vice versa. kUseMmap is accepted; the index is always copied
// into device memory.
#ifndef NSPARSE_B200_INDEX_IO_H
#define NSPARSE_B200_INDEX_IO_H

#include <cstddef>
#include <cstdint>

#include "nsparse/index.h"

namespace nsparse {

enum IndexIoFlag {
    kUseMmap = 0x0001,
};

class IOReader {
public:
    virtual ~IOReader() = default;
    virtual size_t read(void* ptr, size_t size, size_t nitems) = 0;
    virtual size_t pos() const = 0;
    virtual void close() {}
};

class IOWriter {
public:
    virtual ~IOWriter() = default;
    virtual void write(const void* ptr, size_t size, size_t nitems) = 0;
    virtual size_t pos() const = 0;
    virtual void close() {}
};

void write_index(Index* index, const char* file_name);
void write_index(Index* index, IOWriter* io_writer);
Index* read_index(const char* file_name, int io_flags = 0);
Index* read_index(IOReader* io_reader, int io_flags = 0);

}  // namespace nsparse

#endif
