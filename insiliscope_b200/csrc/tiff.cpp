// The movie file the reference's CLI writes (TiffWriter, cli/tiff_writer.h), byte for byte: a little-endian baseline
// TIFF of one uncompressed grey page per frame (16-bit ADU or 32-bit float), or past the classic format's 4 GB a
// BigTIFF (magic 43, 64-bit offsets); plus pages straight from device memory.
//
// The layout every reader and the reference's files share (tiff_writer.h:31-199), restated:
//   header   classic "II" 42 u16, first-IFD offset u32 (at 4);  BigTIFF "II" 43 u16, 8 u16, 0 u16, first offset u64 (8)
//   a page   [samples][description + NUL, when one is given][one 0 byte when the end is odd][IFD]
//   IFD      entry count (u16 | u64), entries in tag order, next-IFD offset (u32 | u64) = 0; the previous page's
//            next-IFD field (the header's first for page 1) is patched to this IFD. Entries: 256 width LONG,
//            257 height LONG, 258 bits SHORT, 259 compression SHORT 1, 262 photometric SHORT 1, [270 description
//            ASCII], 273 strip offset, 277 samples/pixel SHORT 1, 278 rows/strip LONG h, 279 strip bytes, [339 sample
//            format SHORT 3 for float]; 273/279 are LONG in a classic file and LONG8 in a BigTIFF. A classic entry is
//            tag u16, type u16, count u32, value u32 (a SHORT in its low half); a BigTIFF entry tag u16, type u16,
//            count u64, then 8 value bytes: SHORT u16 + 6 zero bytes, LONG u32 + 4, LONG8 u64. A description that
//            fits the value field (4 or 8 bytes with its NUL) sits there, else at its offset.
//   BigTIFF  when asked, or when the expected size + 64 MB reaches 2^32 - 1; a classic file that would pass 2^32 - 1
//            anyway is refused page by page, never written with wrapped offsets.
//   strips   a page may be written with only its first rows, the rest a hole (the file's zeros) that later row
//            writes fill in place: the finished file is the one whole-page writes make.
// Every page is flushed and checked, so a full disk shows at the page it hit, with the reference's messages.

#include "iscu_internal.h"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

struct iscu_tiff
{
   std::FILE* f = nullptr;
   std::string path, error;
   bool big = false;
   uint64_t linkAt = 4;   // where the next page's IFD offset goes
   uint64_t end = 0;      // bytes in the file
   uint64_t pages = 0;
   std::vector<uint64_t> dataAt;   // each page's samples (row writes)
   std::vector<uint32_t> pageW, pageH;
};

namespace {

constexpr uint64_t kClassicEnd = 0xFFFFFFFFull;

int SeekTo(std::FILE* f, uint64_t at) { return fseeko(f, static_cast<off_t>(at), SEEK_SET); }

void Failed(iscu_tiff* t, const char* what)
{
   const int e = errno;
   t->error = "cannot write " + t->path + " (" + what + ", page " + std::to_string(t->pages + 1) + ", " +
              std::to_string(t->end / 1000000) + " MB written): " + (e ? std::strerror(e) : "write error");
}

void Bytes(iscu_tiff* t, const void* p, size_t n)
{
   if (!t->error.empty())
      return;
   if (n && std::fwrite(p, 1, n, t->f) != n)
      Failed(t, "writing");
   t->end += n;
}

template <class T>
void Le(iscu_tiff* t, T v)   // the host is little-endian (x86-64, aarch64), as the format
{
   Bytes(t, &v, sizeof v);
}

struct Entry
{
   uint16_t tag, type;
   uint64_t count, value;
};

int Status(iscu_tiff* t)
{
   if (t->error.empty())
      return ISCU_OK;
   return iscu::Fail(ISCU_ERR_IO, t->error);
}

// One page: `given` of its pageBytes sample bytes from px (the rest a hole), then its description and IFD.
int WritePage(iscu_tiff* t, const void* px, uint32_t sampleBytes, uint16_t sampleFormat, uint32_t w, uint32_t h,
              const char* desc, uint64_t given)
{
   if (!t->f || !t->error.empty())
      return Status(t);
   const uint64_t pageBytes = static_cast<uint64_t>(w) * h * sampleBytes;
   if (given > pageBytes)
      given = pageBytes;
   const size_t dlen = desc ? std::strlen(desc) : 0;
   const uint32_t descBytes = dlen ? static_cast<uint32_t>(dlen) + 1 : 0;   // with its NUL
   if (!t->big && t->end + pageBytes + descBytes + 2 + 2 + 11 * 12 + 4 > kClassicEnd)
   {
      t->error = "cannot write " + t->path + ": page " + std::to_string(t->pages + 1) +
                 " would pass the 4 GB of a classic TIFF (the file was expected to be smaller; insiliscope_cli "
                 "--bigtiff 1 writes a BigTIFF)";
      return Status(t);
   }
   const uint64_t dataAt = t->end;
   errno = 0;
   Bytes(t, px, static_cast<size_t>(given));
   if (given < pageBytes)
   {
      t->end += pageBytes - given;
      if (t->error.empty() && SeekTo(t->f, t->end) != 0)
      {
         Failed(t, "seeking");
         return Status(t);
      }
   }
   t->dataAt.push_back(dataAt);
   t->pageW.push_back(w);
   t->pageH.push_back(h);
   uint64_t descAt = 0;
   if (descBytes)
   {
      descAt = t->end;
      Bytes(t, desc, descBytes);
   }
   if (t->end & 1)
      Le<uint8_t>(t, 0);
   const uint64_t ifdAt = t->end;
   const uint16_t offsetType = t->big ? 16 : 4;   // LONG8 : LONG
   Entry e[11];
   int n = 0;
   e[n++] = {256, 4, 1, w};
   e[n++] = {257, 4, 1, h};
   e[n++] = {258, 3, 1, sampleBytes * 8ull};
   e[n++] = {259, 3, 1, 1};
   e[n++] = {262, 3, 1, 1};
   if (descBytes)
      e[n++] = {270, 2, descBytes, descAt};
   e[n++] = {273, offsetType, 1, dataAt};
   e[n++] = {277, 3, 1, 1};
   e[n++] = {278, 4, 1, h};
   e[n++] = {279, offsetType, 1, pageBytes};
   if (sampleFormat != 1)
      e[n++] = {339, 3, 1, sampleFormat};
   const size_t inPlace = t->big ? 8 : 4;   // value-field bytes
   if (t->big)
      Le<uint64_t>(t, static_cast<uint64_t>(n));
   else
      Le<uint16_t>(t, static_cast<uint16_t>(n));
   for (int i = 0; i < n; ++i)
   {
      Le<uint16_t>(t, e[i].tag);
      Le<uint16_t>(t, e[i].type);
      if (t->big)
         Le<uint64_t>(t, e[i].count);
      else
         Le<uint32_t>(t, static_cast<uint32_t>(e[i].count));
      if (e[i].tag == 270 && descBytes <= inPlace)
      {
         uint8_t v[8] = {};
         std::memcpy(v, desc, descBytes);
         Bytes(t, v, inPlace);
      }
      else if (!t->big)
         Le<uint32_t>(t, static_cast<uint32_t>(e[i].value));   // a SHORT in the low half
      else if (e[i].type == 3)
      {
         Le<uint16_t>(t, static_cast<uint16_t>(e[i].value));
         Le<uint16_t>(t, 0);
         Le<uint32_t>(t, 0);
      }
      else if (e[i].type == 4)
      {
         Le<uint32_t>(t, static_cast<uint32_t>(e[i].value));
         Le<uint32_t>(t, 0);
      }
      else
         Le<uint64_t>(t, e[i].value);
   }
   const uint64_t nextAt = t->end;
   if (t->big)
      Le<uint64_t>(t, 0);
   else
      Le<uint32_t>(t, 0);
   if (!t->error.empty())
      return Status(t);
   // the previous page's (or the header's) link to this IFD
   if (SeekTo(t->f, t->linkAt) != 0)
   {
      Failed(t, "seeking");
      return Status(t);
   }
   const uint64_t keep = t->end;
   if (t->big)
      Le<uint64_t>(t, ifdAt);
   else
      Le<uint32_t>(t, static_cast<uint32_t>(ifdAt));
   t->end = keep;
   if (std::fseek(t->f, 0, SEEK_END) != 0)
   {
      Failed(t, "seeking");
      return Status(t);
   }
   if (std::fflush(t->f) != 0)
   {
      Failed(t, "writing");
      return Status(t);
   }
   t->linkAt = nextAt;
   if (!t->error.empty())
      return Status(t);
   if (std::ferror(t->f))
   {
      Failed(t, "writing");
      return Status(t);
   }
   ++t->pages;
   return ISCU_OK;
}

} // namespace

using namespace iscu;

extern "C" {

uint64_t iscu_tiff_bytes(uint64_t w, uint64_t h, uint64_t pages, uint64_t bytes_per_sample, uint64_t desc_bytes)
{
   return 16 + pages * (w * h * bytes_per_sample + 8 + 8 + 13 * 20 + 8) + desc_bytes + 2;
}

int iscu_tiff_open(const char* path, uint64_t expected_bytes, int32_t big_tiff, iscu_tiff** out)
{
   ClearError();
   if (!path || !out)
      return Fail(ISCU_ERR_ARG, "null argument");
   *out = nullptr;
   std::unique_ptr<iscu_tiff> t(new iscu_tiff());
   t->path = path;
   t->big = big_tiff != 0 || expected_bytes + (64ull << 20) >= kClassicEnd;
   t->f = std::fopen(path, "wb");
   if (!t->f)
      return Fail(ISCU_ERR_IO, "cannot open " + t->path + " for writing: " + std::strerror(errno));
   if (t->big)
   {
      const uint8_t hdr[16] = {'I', 'I', 43, 0, 8, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
      Bytes(t.get(), hdr, 16);
      t->linkAt = 8;
   }
   else
   {
      const uint8_t hdr[8] = {'I', 'I', 42, 0, 0, 0, 0, 0};
      Bytes(t.get(), hdr, 8);
      t->linkAt = 4;
   }
   if (!t->error.empty())
   {
      std::fclose(t->f);
      return Fail(ISCU_ERR_IO, t->error);
   }
   *out = t.release();
   return ISCU_OK;
}

int iscu_tiff_info(iscu_tiff* t, int32_t* big, uint64_t* pages, uint64_t* bytes)
{
   if (!t)
      return Fail(ISCU_ERR_ARG, "null writer");
   if (big)
      *big = t->big ? 1 : 0;
   if (pages)
      *pages = t->pages;
   if (bytes)
      *bytes = t->end;
   return ISCU_OK;
}

int iscu_tiff_page_u16(iscu_tiff* t, const uint16_t* px, uint32_t w, uint32_t h, const char* desc)
{
   ClearError();
   if (!t || (!px && w && h))
      return Fail(ISCU_ERR_ARG, "null argument");
   return WritePage(t, px, 2, 1, w, h, desc, ~0ull);
}

int iscu_tiff_page_f32(iscu_tiff* t, const float* px, uint32_t w, uint32_t h, const char* desc)
{
   ClearError();
   if (!t || (!px && w && h))
      return Fail(ISCU_ERR_ARG, "null argument");
   return WritePage(t, px, 4, 3, w, h, desc, ~0ull);
}

int iscu_tiff_page_rows(iscu_tiff* t, const uint16_t* px, uint32_t rows, uint32_t w, uint32_t h, const char* desc)
{
   ClearError();
   if (!t || (!px && rows && w))
      return Fail(ISCU_ERR_ARG, "null argument");
   return WritePage(t, px, 2, 1, w, h, desc, static_cast<uint64_t>(rows < h ? rows : h) * w * 2);
}

int iscu_tiff_rows(iscu_tiff* t, uint64_t page, uint32_t y0, uint32_t rows, const uint16_t* px)
{
   ClearError();
   if (!t || (!px && rows))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (!t->f || !t->error.empty())
      return Status(t);
   if (page >= t->pages || static_cast<uint64_t>(y0) + rows > t->pageH[page])
   {
      t->error = "cannot write " + t->path + ": rows " + std::to_string(y0) + ".." + std::to_string(y0 + rows) +
                 " of page " + std::to_string(page + 1) + " are not in it";
      return Status(t);
   }
   const uint64_t keep = t->end, row = static_cast<uint64_t>(t->pageW[page]) * 2;
   errno = 0;
   if (SeekTo(t->f, t->dataAt[page] + y0 * row) != 0)
   {
      Failed(t, "seeking");
      return Status(t);
   }
   Bytes(t, px, static_cast<size_t>(rows * row));
   t->end = keep;
   if (SeekTo(t->f, t->end) != 0)
   {
      Failed(t, "seeking");
      return Status(t);
   }
   if (std::fflush(t->f) != 0 || std::ferror(t->f))
   {
      Failed(t, "writing");
      return Status(t);
   }
   return Status(t);
}

int iscu_tiff_pages_dev(iscu_tiff* t, iscu_ctx* ctx, const uint16_t* frames_dev, uint32_t n_frames, uint32_t w,
                        uint32_t h, const char* first_desc)
{
   ClearError();
   if (!t || !ctx || (n_frames && !frames_dev))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (!n_frames)
      return ISCU_OK;
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   const size_t frameBytes = static_cast<size_t>(w) * h * 2;
   // chunks of whole frames, about 8 MB each, two in flight: the copy of chunk k + 1 runs while chunk k is written.
   // The two page-locked halves belong to the context and serve all its writers.
   const uint32_t per = static_cast<uint32_t>(std::max<size_t>(1, (8u << 20) / std::max<size_t>(1, frameBytes)));
   for (int i = 0; i < 2; ++i)
   {
      ISCU_CK(ctx->fileStage[i].Reserve(per * frameBytes));
      if (!ctx->fileCopied[i])
         ISCU_CK(cudaEventCreateWithFlags(&ctx->fileCopied[i], cudaEventDisableTiming));
   }
   if (!ctx->download)
      ISCU_CK(cudaStreamCreateWithFlags(&ctx->download, cudaStreamNonBlocking));
   // the frames are ready after the work enqueued so far on the context's stream
   cudaEvent_t ready;
   ISCU_CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
   cudaError_t e = cudaEventRecord(ready, ctx->stream);
   if (e == cudaSuccess)
      e = cudaStreamWaitEvent(ctx->download, ready, 0);
   cudaEventDestroy(ready);
   ISCU_CK(e);
   const uint32_t chunks = (n_frames + per - 1) / per;
   auto enqueue = [&](uint32_t c) -> cudaError_t {
      const uint32_t f0 = c * per, nf = std::min(per, n_frames - f0);
      cudaError_t r = cudaMemcpyAsync(ctx->fileStage[c & 1].p, frames_dev + static_cast<size_t>(f0) * w * h,
                                      nf * frameBytes, cudaMemcpyDeviceToHost, ctx->download);
      return r == cudaSuccess ? cudaEventRecord(ctx->fileCopied[c & 1], ctx->download) : r;
   };
   ISCU_CK(enqueue(0));
   for (uint32_t c = 0; c < chunks; ++c)
   {
      if (c + 1 < chunks)
         ISCU_CK(enqueue(c + 1));   // into the other half, written out by the previous iteration
      ISCU_CK(cudaEventSynchronize(ctx->fileCopied[c & 1]));
      const uint32_t f0 = c * per, nf = std::min(per, n_frames - f0);
      const uint16_t* px = static_cast<const uint16_t*>(ctx->fileStage[c & 1].p);
      for (uint32_t k = 0; k < nf; ++k)
      {
         const int rc = WritePage(t, px + static_cast<size_t>(k) * w * h, 2, 1, w, h,
                                  f0 + k == 0 ? first_desc : nullptr, ~0ull);
         if (rc != ISCU_OK)
         {
            cudaStreamSynchronize(ctx->download);   // no copy into the staging after the writer moves on
            return rc;
         }
      }
   }
   return ISCU_OK;
}

int iscu_tiff_close(iscu_tiff* t)
{
   ClearError();
   if (!t)
      return ISCU_OK;
   bool closed = true;
   if (t->f)
      closed = std::fclose(t->f) == 0;
   t->f = nullptr;
   if (!closed && t->error.empty())
      Failed(t, "closing it");
   const std::string err = t->error;
   delete t;
   return err.empty() ? ISCU_OK : Fail(ISCU_ERR_IO, err);
}

} // extern "C"
