// The linear revaluation of a group of netting sets as a matrix product: host side.
//
// On a date, every linear term of every netting set of a scenario is a coefficient times one of a few shared
// functions of the path's risk factors: a domestic zero bond 2^(b x), a floating coupon's fixing times its payment
// bond, a foreign bond times its exchange rate S_a 2^(b_f x_f), an exchange rate S_a, or -- one column each -- an
// option's Black price.  Across a book of netting sets these basis functions are far fewer than the terms (bonds of
// one maturity are one function for every netting set), so the netted values of a tile of paths are
//     V[netting set][path] = sum_k C[netting set][k] Phi[path][k]
// with C known at upload.  buildBasis lowers the plans of one group (at most 128 netting sets sharing a scenario,
// reporting dates and margin-call dates) into the tables of basisRevalueKernel:
//   - per date: its k-groups (8 columns of one type each), the fixings it sets and its chunks of 64 columns;
//   - per chunk: C as two FP16 images (hi, lo = the rounding residue of hi), 128 rows in the tensor core's
//     K-major layout, the coefficients of each (date, netting set) scaled by a power of two 2^-s into the FP16
//     range (scale[date][row] = 2^s), and each column's by the inverse of its own scale `mult`;
//   - the fixings a coupon column reads, given a shared-memory slot for their lifetime.
// Plans with other terms, non-cash collateral, longer margin-call look-backs or per-path rows besides the
// exposure rows are not lowered here (the term-by-term kernel runs them).
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace zk {

constexpr int kBasisRows = 128;       // netting sets per group: the MMA's M and TMEM lanes
constexpr int kBasisPaths = 128;      // paths per CTA: the MMA's N
constexpr int kBasisChunkKg = 8;      // k-groups (of 8 columns) per chunk: 64 columns, 4 MMA K-steps
constexpr int kBasisMaxFix = 64;      // fixings live at once (shared-memory slots of 128 paths)
constexpr int kBasisDateWords = 12;   // words per date record
constexpr float kCouponScale = 64.0f; // fixings are kept times 64 (exact): coupon columns of about one
constexpr float kOptionScale = 16.0f; // option prices times 16
constexpr int kBasisOptWords = 12;    // floats per option record (appendOption)

enum BasisColumn : uint32_t {
  kColBond = 0,           // 2^(b x)
  kColCoupon = 1,         // 64 fix[sel] 2^(b x)
  kColForeign = 2,        // S_sel 2^(b x_f[sel])
  kColSpot = 3,           // S_sel
  kColOption = 4,         // 16 Black price of option record sel (a domestic bond numeraire)
  kColForeignOption = 5,  // 16 Black price of a foreign-rate option record sel
};

// One k-group: 8 columns of one type (64 bytes, read with four 16-byte loads).
struct BasisKg {
  float b[8];        // exponent coefficients, -B log2 e
  uint16_t sel[8];   // fixing slot, asset (the k-group's one asset), or option record (relative to the date's first)
  uint32_t type;
  float mult;        // the columns' scale (1, 64 or 16): C is divided by it on the host
  uint32_t pad[2];
};
static_assert(sizeof(BasisKg) == 64, "BasisKg is four 16-byte loads");

// Per date: firstChunk, numChunks, firstKg, numKg, fixBegin, fixEnd, optBegin, callIndex, reportingSlot, the next
// reporting date (nT: none), the previous date's numChunks, the number of option records.
enum BasisDateWord : int {
  bdChunk = 0, bdChunks = 1, bdKg = 2, bdKgs = 3, bdFixBegin = 4, bdFixEnd = 5, bdOpt = 6, bdCall = 7, bdRep = 8,
  bdNextRep = 9, bdPrevChunks = 10, bdOpts = 11,
};
// The kernel's shared memory: the basis and coefficient chunk buffers (128 KB), three dates' staging, two dates'
// k-groups and option records (copied a date ahead), and the fixings' slots; at most 227 KB.
constexpr uint32_t kBasisStageBytes = (3 * 4 * kBasisPaths + 16) * 4;
constexpr uint32_t kBasisFixedSmem = 4 * kBasisPaths * 64 * 2 + 4 * kBasisRows * 64 * 2 + 3 * kBasisStageBytes;
constexpr uint32_t kBasisMaxSmem = 227 * 1024;
inline uint32_t basisSmemBytes(uint32_t descBytes, uint32_t fixSlots) {
  return kBasisFixedSmem + 2 * descBytes + fixSlots * kBasisPaths * 4;
}

// One netting set of a group: its plan's tables as the reference lays them out.
struct BasisPlanIn {
  const float* terms;       // [nTerms][8]
  const uint32_t* indices;  // term starts [nT + 1], margin-call indices at offCall, reporting slots at offRep
  uint32_t nT, nTerms, offCall, offRep;
};

struct BasisImage {
  uint32_t numNs = 0, nT = 0, numFixSlots = 0, numChunks = 0;
  std::vector<uint32_t> dates;      // [nT][kBasisDateWords]
  std::vector<BasisKg> kgs;         // k-groups of every date, in date order
  std::vector<float> options;       // [*][kBasisOptWords]: the option terms, as the kernel prices them
  std::vector<float> fixings;       // [*][4]: A, b, 1 / c, slot
  std::vector<uint32_t> chunks;     // [numChunks][2]: byte offset of the chunk's images in blob, K-steps of 16
  std::vector<uint16_t> blob;       // per chunk: hi image, then lo image (steps * 2 k-groups * 128 rows * 8 halves)
  std::vector<float> scale;         // [nT][kBasisRows]: 2^s
  uint64_t linearTerms = 0;         // the plans' linear terms (bonds, coupons, forwards) and options, all dates
  uint64_t columns = 0;             // basis columns over all dates (padding included)
  uint32_t descBytes = 0;           // the largest date's k-groups and option records, rounded up to 1 KB
};

// Runs fn(0) .. fn(n - 1), possibly on several host threads.
using ParallelFor = std::function<void(size_t n, const std::function<void(size_t)>& fn)>;

// Lowers a group (its dates on `parallel`'s threads when given); returns false with a reason when a plan of the
// group cannot run on the basis kernel.
bool buildBasis(const std::vector<BasisPlanIn>& plans, BasisImage& out, std::string& why,
                const ParallelFor& parallel = nullptr);

// Host check of a lowered group along one path of factor values x[j], S[j][4], xf[j][2] (j < nT): on every date
// the value of every netting set's basis terms, once from the image as the kernel combines it (each column's
// function times the FP16 hi + lo coefficients, times the date's scale; fixings through the image's slots) and
// once term by term from the plans' own records (fixings per swap slot), both in double.  Returns the largest
// |difference| of a netting set over the dates relative to the largest gross sum sum_k |C_k Phi_k| of its basis
// terms over the dates (the scale the FP16 hi + lo coefficients' rounding, about 2^-22, is relative to).
double basisCheck(const std::vector<BasisPlanIn>& plans, const BasisImage& img, const double* x, const double* S,
                  const double* xf);

}  // namespace zk
