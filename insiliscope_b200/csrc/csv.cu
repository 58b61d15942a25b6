// The ground-truth tables' text on sm_100a: numbers as sim::AppendCsvNumber writes them (CsvNumber.cpp:13-32, printf
// of "%.<p>f" / "%.<p>g" at most 47 characters, nothing for NaN and infinities; csv_format.cuh) and integers as
// GroundTruth.cpp's Int (std::to_chars), formatted a value per thread; and whole numeric tables in the layout of
// GroundTruth::FramesCsv (GroundTruth.cpp:307-339): a row is its cells joined by ',' and ended by '\n'.
//
// A table is two passes over its rows with a scan between them, so no cell text is stored: pass 1 formats each
// row's cells (a thread per row, reading the column-major table coalesced) to count its bytes and sums them per block
// of 1024 rows; one thread scans the block sums; pass 2 formats each row again into its place in a shared-memory span
// of 256 rows, which the CTA then stores with aligned 16-byte stores (writes past the caller's capacity are dropped
// and reported).

#include "iscu_internal.h"
#include "csv_format.cuh"

#include <cstring>

namespace iscu {
namespace {

constexpr int kRows = 1024;   // rows per block of the table passes (threads per CTA)
constexpr int kMaxCols = 64;

struct ColFmt
{
   char kind;   // 'f', 'g' (AppendCsvNumber) or 'd' (an integer: std::to_chars of the value as a long long)
   int8_t prec;
};

struct Fmts
{
   ColFmt c[kMaxCols];
};

// "%.<p>f", "%.<p>g" (the forms AppendCsvNumber reads: fmt[2] the precision, fmt[3] the style) or "%d".
bool ParseFmt(const char* fmt, ColFmt& f)
{
   if (!fmt)
      return false;
   if (std::strcmp(fmt, "%d") == 0)
   {
      f = {'d', 0};
      return true;
   }
   if (std::strlen(fmt) == 4 && fmt[0] == '%' && fmt[1] == '.' && fmt[2] >= '0' && fmt[2] <= '9' &&
       (fmt[3] == 'f' || fmt[3] == 'g'))
   {
      f = {fmt[3], static_cast<int8_t>(fmt[2] - '0')};
      return true;
   }
   return false;
}

__device__ __forceinline__ int FormatCell(double v, ColFmt f, char* out)
{
   if (f.kind != 'd')
      return csv::Format(v, f.kind, f.prec, out);
   long long x = static_cast<long long>(v);
   unsigned long long a = x < 0 ? 0ull - static_cast<unsigned long long>(x) : static_cast<unsigned long long>(x);
   char rev[20];
   int n = 0;
   do
   {
      rev[n++] = static_cast<char>('0' + a % 10);
      a /= 10;
   } while (a);
   int len = 0;
   if (x < 0)
      out[len++] = '-';
   while (n)
      out[len++] = rev[--n];
   return len;
}

__global__ void CsvNumbersKernel(const double* __restrict__ v, uint32_t n, ColFmt f, char* __restrict__ fields,
                                 uint8_t* __restrict__ lens)
{
   const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n)
      return;
   char buf[48];
   const int len = FormatCell(v[i], f, buf);
   char* o = fields + static_cast<size_t>(i) * 48;
   for (int j = 0; j < 48; ++j)
      o[j] = j < len ? buf[j] : 0;
   lens[i] = static_cast<uint8_t>(len);
}

// Pass 1: each row's bytes (cells, commas, newline), and their sum per block of kRows rows.
__global__ void __launch_bounds__(kRows) CsvRowLengthsKernel(const double* __restrict__ cols, uint32_t nRows,
                                                            uint32_t nCols, Fmts f, uint32_t* __restrict__ rowLen,
                                                            unsigned long long* __restrict__ blockSum)
{
   __shared__ unsigned long long warpSum[kRows / 32];
   const uint32_t r = blockIdx.x * kRows + threadIdx.x;
   uint32_t len = 0;
   if (r < nRows)
   {
      char buf[48];
      len = nCols;   // nCols - 1 commas and the newline
      for (uint32_t c = 0; c < nCols; ++c)
         len += FormatCell(cols[static_cast<size_t>(c) * nRows + r], f.c[c], buf);
      rowLen[r] = len;
   }
   unsigned long long s = len;
   for (int o = 16; o; o >>= 1)
      s += __shfl_down_sync(0xFFFFFFFFu, s, o);
   if ((threadIdx.x & 31) == 0)
      warpSum[threadIdx.x >> 5] = s;
   __syncthreads();
   if (threadIdx.x == 0)
   {
      unsigned long long t = 0;
      for (int w = 0; w < kRows / 32; ++w)
         t += warpSum[w];
      blockSum[blockIdx.x] = t;
   }
}

// The block sums' exclusive scan in place, the total at blockSum[nBlocks]; one thread (a few thousand blocks).
__global__ void CsvScanBlocksKernel(unsigned long long* blockSum, uint32_t nBlocks)
{
   unsigned long long t = 0;
   for (uint32_t b = 0; b < nBlocks; ++b)
   {
      const unsigned long long v = blockSum[b];
      blockSum[b] = t;
      t += v;
   }
   blockSum[nBlocks] = t;
}

// Pass 2: each row at its offset, formatted again. A CTA takes kSpan rows of a block (their offset: the block's, plus
// the rows before them in the block), lays its rows out in shared memory at the output's 16-byte phase, and the CTA
// stores the span with aligned 16-byte stores (bytes at its two ends, and past the caller's capacity, one at a time).
// A span longer than the staging buffer is written straight from each thread.
constexpr int kSpan = 256;                     // rows (threads) per CTA of pass 2
constexpr int kStage = 64 * 1024;              // staging bytes per CTA

__global__ void __launch_bounds__(kSpan) CsvWriteRowsKernel(const double* __restrict__ cols, uint32_t nRows,
                                                           uint32_t nCols, Fmts f,
                                                           const uint32_t* __restrict__ rowLen,
                                                           const unsigned long long* __restrict__ blockOff,
                                                           char* __restrict__ out, unsigned long long cap)
{
   extern __shared__ uint4 stage4[];
   char* stage = reinterpret_cast<char*>(stage4);
   __shared__ unsigned long long warpSum[kSpan / 32];
   __shared__ unsigned long long spanBefore[kSpan / 32];
   const uint32_t block = blockIdx.x / (kRows / kSpan), sub = blockIdx.x % (kRows / kSpan);
   const uint32_t blockRow0 = block * kRows;
   const uint32_t r = blockRow0 + sub * kSpan + threadIdx.x;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   // the block's rows before this span: sub * kSpan lengths
   unsigned long long pre = 0;
   for (uint32_t i = threadIdx.x; i < sub * kSpan; i += kSpan)
      pre += blockRow0 + i < nRows ? rowLen[blockRow0 + i] : 0u;
   for (int o = 16; o; o >>= 1)
      pre += __shfl_down_sync(0xFFFFFFFFu, pre, o);
   if (lane == 0)
      spanBefore[warp] = pre;
   // this row's offset inside the span: an inclusive scan inside the warp, then across the warps
   const unsigned long long len = r < nRows ? rowLen[r] : 0;
   unsigned long long s = len;
   for (int o = 1; o < 32; o <<= 1)
   {
      const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o)
         s += y;
   }
   if (lane == 31)
      warpSum[warp] = s;
   __syncthreads();
   unsigned long long before = 0, spanBytes = 0, spanAt = blockOff[block];
   for (int w = 0; w < kSpan / 32; ++w)
   {
      before += w < warp ? warpSum[w] : 0u;
      spanBytes += warpSum[w];
      spanAt += spanBefore[w];
   }
   const unsigned long long rowAt = before + s - len;   // inside the span
   const int phase = static_cast<int>(spanAt & 15u);
   const bool staged = phase + spanBytes <= static_cast<unsigned long long>(kStage) &&
                       (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
   if (r < nRows)
   {
      char buf[48];
      unsigned long long at = staged ? phase + rowAt : spanAt + rowAt;
      char* dst = staged ? stage : out;
      const unsigned long long lim = staged ? ~0ull : cap;
      for (uint32_t c = 0; c < nCols; ++c)
      {
         const int n = FormatCell(cols[static_cast<size_t>(c) * nRows + r], f.c[c], buf);
         for (int j = 0; j < n; ++j, ++at)
            if (at < lim)
               dst[at] = buf[j];
         if (at < lim)
            dst[at] = c + 1 < nCols ? ',' : '\n';
         ++at;
      }
   }
   if (!staged)
      return;
   __syncthreads();
   // stage[phase + k] is out[spanAt + k]; the 16-byte chunks of out from spanAt - phase
   const unsigned long long g0 = spanAt - phase, g1 = spanAt + spanBytes;
   const uint32_t chunks = static_cast<uint32_t>((g1 - g0 + 15) / 16);
   uint4* out4 = reinterpret_cast<uint4*>(out + g0);
   for (uint32_t k = threadIdx.x; k < chunks; k += kSpan)
   {
      const unsigned long long c0 = g0 + 16ull * k;
      if (c0 >= spanAt && c0 + 16 <= g1 && c0 + 16 <= cap)
         out4[k] = stage4[k];
      else
         for (int j = 0; j < 16; ++j)
         {
            const unsigned long long g = c0 + j;
            if (g >= spanAt && g < g1 && g < cap)
               out[g] = stage[16 * k + j];
         }
   }
}

} // namespace
} // namespace iscu

using namespace iscu;

extern "C" {

int iscu_csv_numbers_dev(iscu_ctx* ctx, const double* values_dev, uint32_t n, const char* fmt, char* fields_dev,
                         uint8_t* lengths_dev)
{
   if (!ctx || (n && (!values_dev || !fields_dev || !lengths_dev)))
      return Fail(ISCU_ERR_ARG, "null argument");
   ColFmt f;
   if (!ParseFmt(fmt, f))
      return Fail(ISCU_ERR_ARG, "format: \"%.<digit>f\", \"%.<digit>g\" or \"%d\"");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   if (!n)
      return ISCU_OK;
   CsvNumbersKernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(values_dev, n, f, fields_dev, lengths_dev);
   ISCU_CK_LAUNCH(ctx, "CsvNumbersKernel");
   return ISCU_OK;
}

int iscu_csv_table_dev(iscu_ctx* ctx, const double* columns_dev, uint32_t n_rows, uint32_t n_cols,
                       const char* const* fmts, char* out_dev, uint64_t out_capacity, uint64_t* out_bytes)
{
   if (!ctx || !out_bytes || !fmts || (n_rows && (!columns_dev || (!out_dev && out_capacity))))
      return Fail(ISCU_ERR_ARG, "null argument");
   if (n_cols == 0 || n_cols > kMaxCols)
      return Fail(ISCU_ERR_LIMIT, "a table of 1 to 64 columns");
   Fmts f;
   for (uint32_t c = 0; c < n_cols; ++c)
      if (!ParseFmt(fmts[c], f.c[c]))
         return Fail(ISCU_ERR_ARG, "column " + std::to_string(c) + "'s format: \"%.<digit>f\", \"%.<digit>g\" or "
                                   "\"%d\"");
   std::lock_guard<std::recursive_mutex> lock(ctx->mu);
   ClearError();
   *out_bytes = 0;
   if (!n_rows)
      return ISCU_OK;
   const uint32_t blocks = (n_rows + kRows - 1) / kRows;
   const size_t lenBytes = (static_cast<size_t>(n_rows) * 4 + 255) & ~size_t(255);
   ISCU_CK(ctx->dCsv.Reserve(lenBytes + (static_cast<size_t>(blocks) + 1) * 8));
   uint32_t* rowLen = ctx->dCsv.as<uint32_t>();
   auto* blockSum = reinterpret_cast<unsigned long long*>(ctx->dCsv.as<char>() + lenBytes);
   CsvRowLengthsKernel<<<blocks, kRows, 0, ctx->stream>>>(columns_dev, n_rows, n_cols, f, rowLen, blockSum);
   ISCU_CK_LAUNCH(ctx, "CsvRowLengthsKernel");
   CsvScanBlocksKernel<<<1, 1, 0, ctx->stream>>>(blockSum, blocks);
   ISCU_CK_LAUNCH(ctx, "CsvScanBlocksKernel");
   if (out_capacity)   // (a call that only sizes the text writes nothing)
   {
      ISCU_CK(cudaFuncSetAttribute(CsvWriteRowsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStage));
      CsvWriteRowsKernel<<<blocks * (kRows / kSpan), kSpan, kStage, ctx->stream>>>(columns_dev, n_rows, n_cols, f,
                                                                                  rowLen, blockSum, out_dev,
                                                                                  out_capacity);
      ISCU_CK_LAUNCH(ctx, "CsvWriteRowsKernel");
   }
   unsigned long long total = 0;
   ISCU_CK(cudaMemcpyAsync(&total, blockSum + blocks, 8, cudaMemcpyDeviceToHost, ctx->stream));
   ISCU_CK(cudaStreamSynchronize(ctx->stream));
   *out_bytes = total;
   if (total > out_capacity)
      return Fail(ISCU_ERR_LIMIT, "the table needs " + std::to_string(total) + " bytes, the output holds " +
                                  std::to_string(out_capacity) + " (its first bytes are written)");
   return ISCU_OK;
}

} // extern "C"
