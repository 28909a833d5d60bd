// Harness around the reference's table reader,
// pimdal/main/tpc_h/reader/read_table.cpp (compiled from where it lies;
// nothing copied).  Test infrastructure only: it exposes the reader's
// date_to_int, the packed-date encoding of the TPC-H pipelines' date columns,
// to pin the ingest module's restatement.
#include <parquet/arrow/reader.h>

// read_table.cpp was written against Arrow 12 (the reference's Dockerfile
// pins apache-arrow-12.0.1), whose parquet::arrow::OpenFile also took an out
// parameter; Arrow 24 (the pyarrow wheel here) only returns a Result.  This
// overload gives the older form on top of the newer one.
namespace parquet {
namespace arrow {
inline ::arrow::Status OpenFile(std::shared_ptr<::arrow::io::RandomAccessFile> file,
                                ::arrow::MemoryPool *pool, std::unique_ptr<FileReader> *out) {
  ARROW_ASSIGN_OR_RAISE(*out, OpenFile(std::move(file), pool));
  return ::arrow::Status::OK();
}
}  // namespace arrow
}  // namespace parquet

#include "read_table.cpp"

extern "C" {

// Packs n "YYYY-MM-DD" strings (fixed 10-byte records) with date_to_int.
void pimdal_ref_date_to_int(const char *dates, uint64_t n, int32_t *out) {
  for (uint64_t i = 0; i < n; i++) out[i] = date_to_int(std::string(dates + 10 * i, 10));
}

}  // extern "C"
