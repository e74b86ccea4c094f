// Native BookShelf reader (.aux naming .nodes, .scl, .pl, .nets and .wts).
//
// The reference reads every file line by line through std::istringstream
// (src/io/BookshelfParser.cpp:62-311).  This reader builds the same records
// from whole-file buffers split at line boundaries into pieces that several
// host threads parse at once:
//   * `Fields` accepts exactly what `stream >> std::string`, `stream >> double`
//     and `stream >> std::size_t` accept (libstdc++'s num_get grammar in the
//     classic locale; values correctly rounded, as strtod rounds them);
//   * module and net names go into lock-free open-addressing tables filled by
//     all threads, which also find the first duplicate name in file order;
//   * the .nets structure (a NetDegree record owns the next `degree` non-empty
//     lines, whatever they hold) is resolved by one walk over the header lines
//     only, after which the pin lines are parsed in parallel.
// On malformed input the error raised is the one the reference raises first in
// file order, with the reference's text.
#include "bookshelf.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <charconv>
#include <clocale>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <filesystem>
#include <future>
#include <limits>
#include <locale.h>
#include <memory>
#include <mutex>
#include <optional>
#include <string_view>
#include <thread>
#include <unordered_map>
#include <utility>

#include "common.cuh"
#include "mpgp.h"
#include "workers.hpp"

namespace mpgp {
namespace {

namespace fs = std::filesystem;
using Text = std::string_view;

constexpr double kEpsilon = 1e-9;  // myplacement/core/Geometry.hpp
constexpr int kOrientationUnknown = 8;
constexpr size_t kPieceBytes = 4096;  // smallest piece worth a thread
constexpr size_t kBlock = 4096;       // records per parallel task
constexpr unsigned kDefaultThreads = 32;  // threads <= 0: one per hardware thread, at most this many

[[noreturn]] void parseError(const std::string& message) { fail(MPGP_ERR_PARSE, message); }
[[noreturn]] void invalidArgument(const std::string& message) { fail(MPGP_ERR_INVALID_ARGUMENT, message); }

// ---- characters -------------------------------------------------------------------

// isspace() in the classic locale: what operator>> skips.
inline bool isSpace(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

// withoutComment + trim (BookshelfParser.cpp:15-24): cut at the first '#', then
// strip " \t\r\n" (only those four) from both ends.
Text stripLine(Text line) {
    if (!line.empty()) {
        if (const void* hash = std::memchr(line.data(), '#', line.size())) {
            line = line.substr(0, static_cast<size_t>(static_cast<const char*>(hash) - line.data()));
        }
    }
    const auto trimmed = [](char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n'; };
    size_t b = 0;
    size_t e = line.size();
    while (b < e && trimmed(line[b])) ++b;
    while (e > b && trimmed(line[e - 1])) --e;
    return line.substr(b, e - b);
}

inline bool beginsWith(Text text, Text prefix) {
    return text.size() >= prefix.size() && text.compare(0, prefix.size(), prefix) == 0;
}

inline char upperChar(char c) { return c >= 'a' && c <= 'z' ? static_cast<char>(c - 'a' + 'A') : c; }

// std::toupper over `text`, compared with an upper-case literal.
bool equalsUpper(Text text, Text upper) {
    if (text.size() != upper.size()) return false;
    for (size_t i = 0; i < text.size(); ++i) {
        if (upperChar(text[i]) != upper[i]) return false;
    }
    return true;
}

// upper(text).find(upper) != npos.
bool containsUpper(Text text, Text upper) {
    if (upper.size() > text.size()) return false;
    for (size_t i = 0; i + upper.size() <= text.size(); ++i) {
        if (equalsUpper(text.substr(i, upper.size()), upper)) return true;
    }
    return false;
}

// parseOrientation (PlacementDatabase.cpp:27-38): N S E W FN FS FE FW, else Unknown.
int parseOrientation(Text text) {
    static constexpr Text kNames[] = {"N", "S", "E", "W", "FN", "FS", "FE", "FW"};
    for (int k = 0; k < 8; ++k) {
        if (equalsUpper(text, kNames[k])) return k;
    }
    return kOrientationUnknown;
}

// parsePinDirection (PlacementDatabase.cpp:70-76).
int8_t parsePinDirection(Text text) {
    if (equalsUpper(text, "I") || equalsUpper(text, "INPUT")) return 0;
    if (equalsUpper(text, "O") || equalsUpper(text, "OUTPUT")) return 1;
    if (equalsUpper(text, "B") || equalsUpper(text, "INOUT")) return 2;
    return 3;
}

// ---- numbers ----------------------------------------------------------------------

locale_t classicLocale() {
    static const locale_t locale = newlocale(LC_ALL_MASK, "C", static_cast<locale_t>(nullptr));
    return locale;
}

// The conversion num_get applies to the characters it collected for a double:
// strtod in the classic locale, failing unless every character is used or when
// the value is beyond the double range (an underflow keeps strtod's value).
// std::from_chars rounds exactly as strtod does; strtod_l settles the values
// from_chars reports out of range.
bool convertReal(const char* begin, const char* end, double& out) {
    const char* p = begin;
    if (p < end && *p == '+') ++p;
    double value = 0.0;
    const std::from_chars_result r = std::from_chars(p, end, value);
    if (r.ec == std::errc() && r.ptr == end) {
        out = value;
        return true;
    }
    if (r.ec == std::errc::result_out_of_range && r.ptr == end) {
        const std::string text(begin, end);
        const double v = strtod_l(text.c_str(), nullptr, classicLocale());
        if (std::isinf(v)) return false;
        out = v;
        return true;
    }
    return false;
}

// extractNumbers (BookshelfParser.cpp:37-54), stopping after `wanted` numbers:
// ':' ',' and '\t' read as blanks, and every blank-separated token that
// std::stod consumes whole is a number (a range error makes it not one).
int leadingNumbers(Text line, double* values, int wanted) {
    const auto blank = [](char c) { return isSpace(c) || c == ':' || c == ','; };
    int found = 0;
    size_t p = 0;
    std::string token;
    while (found < wanted) {
        while (p < line.size() && blank(line[p])) ++p;
        if (p == line.size()) break;
        const size_t b = p;
        while (p < line.size() && !blank(line[p])) ++p;
        token.assign(line.data() + b, p - b);
        char* end = nullptr;
        errno = 0;
        const double v = std::strtod(token.c_str(), &end);
        if (end == token.c_str() || errno == ERANGE) continue;
        if (static_cast<size_t>(end - token.c_str()) != token.size()) continue;
        values[found++] = v;
    }
    return found;
}

// One line read field by field the way an std::istringstream over it reads:
// `word` is operator>>(std::string&), `real` operator>>(double&) and `count`
// operator>>(std::size_t&).  A failed read leaves its target unchanged; callers
// stop at the first failure, as a stream's failbit fails every later read.  With
// `colon_is_blank` a ':' reads as a blank (the reference replaces ':' by ' ' in
// pin lines).
class Fields {
public:
    explicit Fields(Text line, bool colon_is_blank = false) : s_(line), colon_(colon_is_blank) {}

    bool word(Text& out) {
        skip();
        if (p_ == s_.size()) return false;
        const size_t b = p_;
        while (p_ < s_.size() && !blank(s_[p_])) ++p_;
        out = s_.substr(b, p_ - b);
        return true;
    }

    // num_get::_M_extract_float: [sign] digits [. digits] [e [sign] digits],
    // an exponent only after a mantissa digit.
    bool real(double& out) {
        skip();
        const size_t n = s_.size();
        const size_t b = p_;
        size_t q = p_;
        if (q < n && (s_[q] == '+' || s_[q] == '-')) ++q;
        bool mantissa = false;
        bool point = false;
        bool exponent = false;
        while (q < n) {
            const char c = s_[q];
            if (c >= '0' && c <= '9') {
                mantissa = true;
                ++q;
            } else if (c == '.' && !point && !exponent) {
                point = true;
                ++q;
            } else if ((c == 'e' || c == 'E') && !exponent && mantissa) {
                exponent = true;
                ++q;
                if (q < n && (s_[q] == '+' || s_[q] == '-')) ++q;
            } else {
                break;
            }
        }
        p_ = q;
        return convertReal(s_.data() + b, s_.data() + q, out);
    }

    // num_get::_M_extract_int for std::size_t: [sign] digits; a value above the
    // maximum fails and a '-' negates modulo 2^64.
    bool count(uint64_t& out) {
        skip();
        const size_t n = s_.size();
        size_t q = p_;
        bool negative = false;
        if (q < n && (s_[q] == '+' || s_[q] == '-')) {
            negative = s_[q] == '-';
            ++q;
        }
        constexpr uint64_t kMax = std::numeric_limits<uint64_t>::max();
        uint64_t value = 0;
        bool digits = false;
        bool overflow = false;
        for (; q < n && s_[q] >= '0' && s_[q] <= '9'; ++q) {
            const uint64_t d = static_cast<uint64_t>(s_[q] - '0');
            digits = true;
            if (overflow || value > (kMax - d) / 10) {
                overflow = true;
            } else {
                value = value * 10 + d;
            }
        }
        p_ = q;
        if (!digits || overflow) return false;
        out = negative ? uint64_t{0} - value : value;
        return true;
    }

private:
    bool blank(char c) const { return isSpace(c) || (colon_ && c == ':'); }
    void skip() {
        while (p_ < s_.size() && blank(s_[p_])) ++p_;
    }

    Text s_;
    bool colon_;
    size_t p_ = 0;
};

// ---- files, pieces and threads ---------------------------------------------------------

struct FileText {
    bool opened = false;
    std::string data;
};

FileText readWhole(const fs::path& path) {
    FileText out;
    std::FILE* file = std::fopen(path.c_str(), "rb");
    if (file == nullptr) return out;
    out.opened = true;
    struct stat info {};
    if (fstat(fileno(file), &info) == 0 && S_ISREG(info.st_mode) && info.st_size > 0) {
        out.data.resize(static_cast<size_t>(info.st_size));
        out.data.resize(std::fread(out.data.data(), 1, out.data.size(), file));
    }
    char buffer[1 << 16];
    for (size_t got; (got = std::fread(buffer, 1, sizeof(buffer), file)) > 0;) out.data.append(buffer, got);
    std::fclose(file);
    return out;
}

// Line ranges [begin, end) of `text` that start and end at line starts.
struct Piece {
    size_t begin, end;
};

std::vector<Piece> linePieces(Text text, int threads) {
    const size_t size = text.size();
    const size_t wanted = std::max<size_t>(1, std::min<size_t>(static_cast<size_t>(threads) * 4, size / kPieceBytes));
    std::vector<Piece> pieces;
    pieces.reserve(wanted);
    size_t begin = 0;
    for (size_t k = 1; k <= wanted; ++k) {
        size_t end = k == wanted ? size : std::max(begin, size / wanted * k);
        if (end < size) {
            const void* newline = std::memchr(text.data() + end, '\n', size - end);
            end = newline != nullptr ? static_cast<size_t>(static_cast<const char*>(newline) - text.data()) + 1 : size;
        }
        pieces.push_back({begin, end});
        begin = end;
    }
    return pieces;
}

// The next line of `text` at `pos` (std::getline: split at '\n', the last line
// may lack one); advances `pos`.
inline Text nextLine(Text text, size_t& pos, size_t end) {
    const void* newline = std::memchr(text.data() + pos, '\n', end - pos);
    const size_t stop = newline != nullptr ? static_cast<size_t>(static_cast<const char*>(newline) - text.data()) : end;
    const Text line = text.substr(pos, stop - pos);
    pos = newline != nullptr ? stop + 1 : end;
    return line;
}

// 1-based number of the line holding byte `offset`.
int64_t lineNumberAt(Text text, size_t offset) {
    return 1 + static_cast<int64_t>(std::count(text.data(), text.data() + offset, '\n'));
}

// ---- names --------------------------------------------------------------------------

uint64_t hashName(Text s) {
    constexpr uint64_t kMul = 0x9E3779B97F4A7C15ull;
    uint64_t h = 0x243F6A8885A308D3ull ^ (s.size() * kMul);
    size_t i = 0;
    for (; i + 8 <= s.size(); i += 8) {
        uint64_t w;
        std::memcpy(&w, s.data() + i, 8);
        h = (h ^ w) * kMul;
        h ^= h >> 29;
    }
    uint64_t w = 0;
    std::memcpy(&w, s.data() + i, s.size() - i);
    h = (h ^ w) * kMul;
    h ^= h >> 32;
    h *= 0xD6E8FEB86659FD93ull;
    h ^= h >> 32;
    return h;
}

// Name -> smallest index with that name.  Open addressing with linear probing;
// a slot holds the upper 32 bits of the hash beside a 32-bit index and every
// thread inserts at once.  When two equal names meet, the larger index is a
// duplicate and the slot keeps the smaller, so once every name is in, the
// smallest index flagged is the first name in file order that repeats an
// earlier one.
class NameTable {
public:
    void build(const std::vector<Text>& names, const Workers& workers) {
        names_ = &names;
        size_t capacity = 16;
        while (capacity < 2 * names.size()) capacity <<= 1;
        mask_ = capacity - 1;
        slots_.reset(new std::atomic<uint64_t>[capacity]);
        workers.blocks(capacity, kBlock, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) slots_[i].store(kEmpty, std::memory_order_relaxed);
        });
        workers.blocks(names.size(), kBlock, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; ++i) insert(static_cast<uint32_t>(i));
        });
    }

    [[nodiscard]] int64_t find(Text name) const { return findHashed(name, hashName(name)); }

    // find() of `count` names into `out`.  The lookups go in groups whose slot,
    // name-record and name-byte loads are each issued for the whole group
    // before any is used, so their cache misses overlap.
    void findMany(const Text* names, int64_t* out, size_t count) const {
        constexpr size_t kGroup = 32;
        uint64_t hash[kGroup];
        uint64_t slot[kGroup];
        for (size_t g = 0; g < count; g += kGroup) {
            const size_t n = std::min(kGroup, count - g);
            for (size_t i = 0; i < n; ++i) {
                hash[i] = hashName(names[g + i]);
                __builtin_prefetch(&slots_[hash[i] & mask_]);
            }
            for (size_t i = 0; i < n; ++i) {
                slot[i] = slots_[hash[i] & mask_].load(std::memory_order_relaxed);
                if (slot[i] != kEmpty) __builtin_prefetch(&(*names_)[static_cast<uint32_t>(slot[i])]);
            }
            for (size_t i = 0; i < n; ++i) {
                if (slot[i] != kEmpty && (slot[i] >> 32) == (hash[i] >> 32)) {
                    __builtin_prefetch((*names_)[static_cast<uint32_t>(slot[i])].data());
                }
            }
            for (size_t i = 0; i < n; ++i) out[g + i] = findHashed(names[g + i], hash[i]);
        }
    }

private:
    [[nodiscard]] int64_t findHashed(Text name, uint64_t h) const {
        for (size_t s = h & mask_;; s = (s + 1) & mask_) {
            const uint64_t cur = slots_[s].load(std::memory_order_relaxed);
            if (cur == kEmpty) return -1;
            if ((cur >> 32) == (h >> 32) && (*names_)[static_cast<uint32_t>(cur)] == name) {
                return static_cast<uint32_t>(cur);
            }
        }
    }

public:
    // The first index whose name occurs at a smaller index, or -1.
    [[nodiscard]] int64_t firstDuplicate() const {
        const int64_t d = first_duplicate_.load();
        return d == kNone ? -1 : d;
    }

private:
    static constexpr uint64_t kEmpty = ~uint64_t{0};
    static constexpr int64_t kNone = std::numeric_limits<int64_t>::max();

    void insert(uint32_t index) {
        const Text name = (*names_)[index];
        const uint64_t h = hashName(name);
        const uint64_t mine = (h >> 32 << 32) | index;
        size_t s = h & mask_;
        uint64_t cur = slots_[s].load(std::memory_order_relaxed);
        for (;;) {
            if (cur == kEmpty) {
                if (slots_[s].compare_exchange_weak(cur, mine, std::memory_order_relaxed)) return;
                continue;  // `cur` now holds what took the slot
            }
            if ((cur >> 32) == (h >> 32) && (*names_)[static_cast<uint32_t>(cur)] == name) {
                const uint32_t other = static_cast<uint32_t>(cur);
                noteDuplicate(std::max(index, other));
                if (index > other) return;
                if (slots_[s].compare_exchange_weak(cur, mine, std::memory_order_relaxed)) return;
                continue;
            }
            s = (s + 1) & mask_;
            cur = slots_[s].load(std::memory_order_relaxed);
        }
    }

    void noteDuplicate(int64_t index) {
        int64_t seen = first_duplicate_.load(std::memory_order_relaxed);
        while (index < seen && !first_duplicate_.compare_exchange_weak(seen, index, std::memory_order_relaxed)) {
        }
    }

    const std::vector<Text>* names_ = nullptr;
    std::unique_ptr<std::atomic<uint64_t>[]> slots_;
    size_t mask_ = 0;
    std::atomic<int64_t> first_duplicate_{kNone};
};

// Concatenates `names` into `blob` with `start` offsets (count + 1).
void storeNames(const std::vector<Text>& names, const Workers& workers, std::string& blob,
                std::vector<int64_t>& start) {
    start.assign(names.size() + 1, 0);
    for (size_t i = 0; i < names.size(); ++i) start[i + 1] = start[i] + static_cast<int64_t>(names[i].size());
    blob.resize(static_cast<size_t>(start.back()));
    workers.blocks(names.size(), kBlock, [&](size_t b, size_t e) {
        for (size_t i = b; i < e; ++i) {
            if (!names[i].empty()) std::memcpy(blob.data() + start[i], names[i].data(), names[i].size());
        }
    });
}

// ---- .aux (BookshelfParser.cpp:313-328) --------------------------------------------------

std::unordered_map<std::string, fs::path> auxFiles(const fs::path& aux_path, Text text) {
    const fs::path directory = aux_path.parent_path();
    std::unordered_map<std::string, fs::path> files;
    size_t pos = 0;
    while (pos < text.size()) {
        const Text line = stripLine(nextLine(text, pos, text.size()));
        const size_t colon = line.find(':');
        if (line.empty() || colon == Text::npos) continue;
        Fields fields(line.substr(colon + 1));
        Text name;
        while (fields.word(name)) {
            const std::string file_name(name);
            const std::string extension = fs::path(file_name).extension().string();
            if (!extension.empty()) files.emplace(extension, directory / file_name);
        }
    }
    return files;
}

// ---- .nodes (BookshelfParser.cpp:62-98) ---------------------------------------------------

struct NodePiece {
    std::vector<Text> names;
    std::vector<double> width, height;
    std::vector<uint8_t> terminal;
    int64_t lines = 0;
    int failure = 0;  // 1 invalid node, 2 invalid NumNodes, 3 invalid NumTerminals
    std::optional<uint64_t> nodes, terminals;
};

void parseNodePiece(Text text, Piece piece, NodePiece& out) {
    size_t pos = piece.begin;
    while (pos < piece.end) {
        const Text line = stripLine(nextLine(text, pos, piece.end));
        ++out.lines;
        if (line.empty() || beginsWith(line, "UCLA")) continue;
        if (beginsWith(line, "NumNodes") || beginsWith(line, "NumTerminals")) {
            const bool nodes = beginsWith(line, "NumNodes");
            double value = 0.0;
            if (leadingNumbers(line, &value, 1) == 0) {
                out.failure = nodes ? 2 : 3;
                return;
            }
            (nodes ? out.nodes : out.terminals) = static_cast<uint64_t>(static_cast<std::size_t>(value));
            continue;
        }
        Fields fields(line);
        Text name;
        double width = 0.0;
        double height = 0.0;
        if (!(fields.word(name) && fields.real(width) && fields.real(height))) {
            out.failure = 1;
            return;
        }
        bool terminal = false;
        for (Text attribute; fields.word(attribute);) {
            if (containsUpper(attribute, "TERMINAL")) terminal = true;
        }
        out.names.push_back(name);
        out.width.push_back(width);
        out.height.push_back(height);
        out.terminal.push_back(terminal ? 1 : 0);
    }
}

void parseNodes(const fs::path& path, Text text, const Workers& workers, Bookshelf& book,
                std::vector<Text>& names, NameTable& table, std::optional<uint64_t> declared[2]) {
    const std::vector<Piece> pieces = linePieces(text, workers.threads());
    std::vector<NodePiece> parsed(pieces.size());
    workers.run(pieces.size(), [&](size_t i) { parseNodePiece(text, pieces[i], parsed[i]); });

    size_t failed = pieces.size();
    for (size_t i = 0; i < parsed.size(); ++i) {
        if (parsed[i].failure != 0) {
            failed = i;
            break;
        }
    }
    const size_t used = failed == pieces.size() ? pieces.size() : failed + 1;
    std::vector<size_t> first(used + 1, 0);
    for (size_t i = 0; i < used; ++i) first[i + 1] = first[i] + parsed[i].names.size();
    const size_t count = first[used];
    if (count > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
        invalidArgument("The engine indexes modules with 32-bit integers.");
    }
    names.resize(count);
    book.width.resize(count);
    book.height.resize(count);
    book.flags.resize(count);
    workers.run(used, [&](size_t i) {
        const NodePiece& p = parsed[i];
        std::copy(p.names.begin(), p.names.end(), names.begin() + static_cast<std::ptrdiff_t>(first[i]));
        std::copy(p.width.begin(), p.width.end(), book.width.begin() + static_cast<std::ptrdiff_t>(first[i]));
        std::copy(p.height.begin(), p.height.end(), book.height.begin() + static_cast<std::ptrdiff_t>(first[i]));
        for (size_t k = 0; k < p.terminal.size(); ++k) {
            book.flags[first[i] + k] = p.terminal[k] != 0 ? (MPGP_MODULE_TERMINAL | MPGP_MODULE_FIXED) : 0;
        }
    });
    table.build(names, workers);

    // PlacementDatabase::addModule (PlacementDatabase.cpp:78-92) checks the size
    // before the name, module by module; a malformed line stops after the modules
    // read before it.
    size_t negative = count;
    for (size_t m = 0; m < count; ++m) {
        if (book.width[m] < 0.0 || book.height[m] < 0.0) {
            negative = m;
            break;
        }
    }
    const int64_t dup = table.firstDuplicate();
    const size_t duplicate = dup < 0 ? count : static_cast<size_t>(dup);
    if (std::min(negative, duplicate) < count) {
        if (negative <= duplicate) {
            invalidArgument("A module cannot have a negative size: " + std::string(names[negative]));
        }
        invalidArgument("Duplicate module name: " + std::string(names[duplicate]));
    }
    if (failed < pieces.size()) {
        int64_t line = parsed[failed].lines;
        for (size_t i = 0; i < failed; ++i) line += parsed[i].lines;
        static const char* const kWhat[] = {"", "invalid node", "invalid NumNodes", "invalid NumTerminals"};
        parseError(path.string() + ": " + kWhat[parsed[failed].failure] + " at line " + std::to_string(line));
    }
    for (const NodePiece& p : parsed) {
        if (p.nodes) declared[0] = p.nodes;
        if (p.terminals) declared[1] = p.terminals;
    }
    book.x.assign(count, 0.0);
    book.y.assign(count, 0.0);
    book.orientation.assign(count, 0);
}

// ---- .scl (BookshelfParser.cpp:100-160) -----------------------------------------------------

void parseScl(const fs::path& path, Text text, Bookshelf& book) {
    bool inside_row = false;
    double bottom = 0.0;
    double height = 0.0;
    double site_width = 1.0;
    double site_spacing = 1.0;
    int orientation = 0;
    int64_t line_number = 0;
    size_t pos = 0;
    while (pos < text.size()) {
        const Text line = stripLine(nextLine(text, pos, text.size()));
        ++line_number;
        if (line.empty() || beginsWith(line, "UCLA") || beginsWith(line, "NumRows")) continue;
        if (beginsWith(line, "CoreRow")) {
            inside_row = true;
            bottom = 0.0;
            height = 0.0;
            site_width = 1.0;
            site_spacing = 1.0;
            orientation = 0;
            continue;
        }
        if (!inside_row) continue;
        if (line == "End") {
            inside_row = false;
            continue;
        }
        double numbers[2] = {0.0, 0.0};
        const auto first = [&](double& field) {
            if (leadingNumbers(line, numbers, 1) > 0) field = numbers[0];
        };
        if (beginsWith(line, "Coordinate")) {
            first(bottom);
        } else if (beginsWith(line, "Height")) {
            first(height);
        } else if (beginsWith(line, "Sitewidth")) {
            first(site_width);
        } else if (beginsWith(line, "Sitespacing")) {
            first(site_spacing);
        } else if (beginsWith(line, "Siteorient")) {
            Fields fields(line);
            Text label;
            Text separator;
            Text value;
            if (fields.word(label) && fields.word(separator) && fields.word(value)) {
                orientation = parseOrientation(value);
            }
        } else if (beginsWith(line, "SubrowOrigin")) {
            if (leadingNumbers(line, numbers, 2) < 2 || height <= kEpsilon || site_spacing <= kEpsilon) {
                parseError(path.string() + ": invalid SubrowOrigin at line " + std::to_string(line_number));
            }
            book.row_bottom.push_back(bottom);
            book.row_height.push_back(height);
            book.row_site_width.push_back(site_width);
            book.row_site_spacing.push_back(site_spacing);
            book.row_x_start.push_back(numbers[0]);
            book.row_site_count.push_back(static_cast<int64_t>(static_cast<std::size_t>(numbers[1])));
            book.row_orientation.push_back(orientation);
        }
    }
    if (book.row_bottom.empty()) parseError(path.string() + ": contains no valid SiteRow records");
    if (book.row_bottom.size() > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
        invalidArgument("The engine indexes rows with 32-bit integers.");
    }
}

// ---- .pl (BookshelfParser.cpp:162-196) ----------------------------------------------------

struct PlRecord {
    int64_t line;        // within the piece
    int8_t orientation;  // -1: unchanged
    uint8_t fixed;
    double x, y;
};

struct PlPiece {
    std::vector<PlRecord> records;
    std::vector<Text> names;
    std::vector<int64_t> module;
    int64_t lines = 0;
    int64_t failed = -1;  // the record naming an unknown module
};

void parsePlPiece(Text text, Piece piece, const NameTable& modules, PlPiece& out) {
    size_t pos = piece.begin;
    while (pos < piece.end) {
        const Text line = stripLine(nextLine(text, pos, piece.end));
        ++out.lines;
        if (line.empty() || beginsWith(line, "UCLA")) continue;
        Fields fields(line);
        Text name;
        PlRecord record{out.lines, -1, 0, 0.0, 0.0};
        if (!(fields.word(name) && fields.real(record.x) && fields.real(record.y))) continue;
        Text token;
        if (fields.word(token)) {
            if (token == ":") {
                Text next;
                if (fields.word(next)) token = next;  // a lone ':' at the end stays the token
            } else if (token.front() == ':') {
                token.remove_prefix(1);
            }
            if (!token.empty()) record.orientation = static_cast<int8_t>(parseOrientation(token));
        }
        for (Text attribute; fields.word(attribute);) {
            if (containsUpper(attribute, "FIXED")) record.fixed = 1;
        }
        out.records.push_back(record);
        out.names.push_back(name);
    }
    out.module.resize(out.names.size());
    modules.findMany(out.names.data(), out.module.data(), out.names.size());
    for (size_t r = 0; r < out.module.size(); ++r) {
        if (out.module[r] < 0) {
            out.failed = static_cast<int64_t>(r);
            return;
        }
    }
}

void parsePl(const fs::path& path, Text text, const Workers& workers, const NameTable& modules, Bookshelf& book) {
    const std::vector<Piece> pieces = linePieces(text, workers.threads());
    std::vector<PlPiece> parsed(pieces.size());
    workers.run(pieces.size(), [&](size_t i) { parsePlPiece(text, pieces[i], modules, parsed[i]); });
    int64_t line = 0;
    for (const PlPiece& p : parsed) {
        if (p.failed >= 0) {
            const size_t r = static_cast<size_t>(p.failed);
            parseError(path.string() + ": position references unknown module '" + std::string(p.names[r]) +
                       "' at line " + std::to_string(line + p.records[r].line));
        }
        line += p.lines;
    }
    // Module::setLowerLeft (PlacementDatabase.hpp:49-51), in file order.
    for (const PlPiece& p : parsed) {
        for (size_t k = 0; k < p.records.size(); ++k) {
            const PlRecord& r = p.records[k];
            const size_t m = static_cast<size_t>(p.module[k]);
            if (r.orientation >= 0) book.orientation[m] = r.orientation;
            if (r.fixed != 0) book.flags[m] |= MPGP_MODULE_FIXED;
            book.x[m] = r.x + book.width[m] * 0.5;
            book.y[m] = r.y + book.height[m] * 0.5;
        }
    }
}

// ---- .nets (BookshelfParser.cpp:198-263) ----------------------------------------------------

// A non-empty line outside a net that the walk must look at: NumNets, NumPins
// or a NetDegree header (parsed here, `ok` false when the header is invalid).
struct NetHeader {
    int64_t rank;  // among the non-empty lines
    int kind;      // 0 NumNets, 1 NumPins, 2 NetDegree
    bool ok;
    uint64_t value;
    Text name;
};

struct NetsPiece {
    int64_t data_lines = 0;
    std::vector<NetHeader> headers;
};

struct PinFailure {
    int64_t pin = std::numeric_limits<int64_t>::max();
    bool unknown = false;  // else: an invalid pin line
    Text module;
};

void parseNets(const fs::path& path, Text text, const Workers& workers, const NameTable& modules, Bookshelf& book,
               std::vector<Text>& net_names, NameTable& net_table, std::optional<uint64_t> declared[2]) {
    const std::vector<Piece> pieces = linePieces(text, workers.threads());
    std::vector<NetsPiece> parsed(pieces.size());
    // Count the non-empty lines of each piece.
    workers.run(pieces.size(), [&](size_t i) {
        size_t pos = pieces[i].begin;
        while (pos < pieces[i].end) {
            if (!stripLine(nextLine(text, pos, pieces[i].end)).empty()) ++parsed[i].data_lines;
        }
    });
    std::vector<int64_t> rank_base(pieces.size() + 1, 0);
    for (size_t i = 0; i < pieces.size(); ++i) rank_base[i + 1] = rank_base[i] + parsed[i].data_lines;
    const int64_t data_lines = rank_base.back();
    // Where each non-empty line starts, and the header candidates.
    std::vector<int64_t> line_start(static_cast<size_t>(data_lines));
    workers.run(pieces.size(), [&](size_t i) {
        int64_t rank = rank_base[i];
        size_t pos = pieces[i].begin;
        while (pos < pieces[i].end) {
            const size_t start = pos;
            const Text line = stripLine(nextLine(text, pos, pieces[i].end));
            if (line.empty()) continue;
            line_start[static_cast<size_t>(rank)] = static_cast<int64_t>(start);
            NetHeader header{rank, -1, true, 0, {}};
            if (beginsWith(line, "NumNets") || beginsWith(line, "NumPins")) {
                header.kind = beginsWith(line, "NumNets") ? 0 : 1;
                double value = 0.0;
                header.ok = leadingNumbers(line, &value, 1) > 0;
                if (header.ok) header.value = static_cast<uint64_t>(static_cast<std::size_t>(value));
            } else if (beginsWith(line, "NetDegree")) {
                header.kind = 2;
                Fields fields(line);
                Text label;
                Text separator;
                header.ok = fields.word(label) && fields.word(separator) && fields.count(header.value) &&
                            fields.word(header.name);
            }
            if (header.kind >= 0) parsed[i].headers.push_back(header);
            ++rank;
        }
    });
    const auto lineText = [&](int64_t rank) {
        size_t pos = static_cast<size_t>(line_start[static_cast<size_t>(rank)]);
        return stripLine(nextLine(text, pos, text.size()));
    };
    const auto lineNumber = [&](int64_t rank) {
        return lineNumberAt(text, static_cast<size_t>(line_start[static_cast<size_t>(rank)]));
    };

    // The walk: a NetDegree record owns the next `degree` non-empty lines.
    std::vector<int64_t> first_rank;
    std::vector<int64_t> pins_read;
    int64_t invalid_header = -1;  // rank of an invalid NetDegree the walk stopped at
    bool truncated = false;       // the last net ran out of lines
    int64_t next = 0;
    for (const NetsPiece& piece : parsed) {
        for (const NetHeader& h : piece.headers) {
            if (h.rank < next || invalid_header >= 0 || truncated) continue;
            if (h.kind < 2) {
                if (h.ok) declared[h.kind] = h.value;
                continue;
            }
            if (!h.ok) {
                invalid_header = h.rank;
                continue;
            }
            const uint64_t available = static_cast<uint64_t>(data_lines - h.rank - 1);
            first_rank.push_back(h.rank + 1);
            net_names.push_back(h.name);
            if (h.value > available) {
                pins_read.push_back(static_cast<int64_t>(available));
                truncated = true;
                continue;
            }
            pins_read.push_back(static_cast<int64_t>(h.value));
            next = h.rank + 1 + static_cast<int64_t>(h.value);
        }
    }
    const size_t nets = net_names.size();
    if (nets > static_cast<size_t>(std::numeric_limits<int32_t>::max())) {
        invalidArgument("The engine indexes nets with 32-bit integers.");
    }
    book.net_pin_start.assign(nets + 1, 0);
    for (size_t n = 0; n < nets; ++n) book.net_pin_start[n + 1] = book.net_pin_start[n] + pins_read[n];
    const int64_t pins = book.net_pin_start.back();
    net_table.build(net_names, workers);

    book.pin_module.resize(static_cast<size_t>(pins));
    book.pin_offset_x.resize(static_cast<size_t>(pins));
    book.pin_offset_y.resize(static_cast<size_t>(pins));
    book.pin_direction.resize(static_cast<size_t>(pins));
    std::mutex failure_lock;
    PinFailure failure;
    workers.blocks(nets, kBlock, [&](size_t b, size_t e) {
        // The block's pins are contiguous: read every line up to the first
        // malformed one, then look the module names up together.
        const int64_t first_pin = book.net_pin_start[b];
        std::vector<Text> names(static_cast<size_t>(book.net_pin_start[e] - first_pin));
        constexpr int64_t kNoFailure = std::numeric_limits<int64_t>::max();
        PinFailure mine;
        int64_t read = 0;
        for (size_t n = b; n < e && mine.pin == kNoFailure; ++n) {
            for (int64_t k = 0; k < pins_read[n]; ++k) {
                const size_t pin = static_cast<size_t>(book.net_pin_start[n] + k);
                Fields fields(lineText(first_rank[n] + k), true);
                Text direction;
                if (!(fields.word(names[read]) && fields.word(direction) && fields.real(book.pin_offset_x[pin]) &&
                      fields.real(book.pin_offset_y[pin]))) {
                    mine = {static_cast<int64_t>(pin), false, {}};
                    break;
                }
                book.pin_direction[pin] = parsePinDirection(direction);
                ++read;
            }
        }
        std::vector<int64_t> module(static_cast<size_t>(read));
        modules.findMany(names.data(), module.data(), module.size());
        for (int64_t k = 0; k < read; ++k) {
            if (module[k] < 0) {
                mine = {first_pin + k, true, names[k]};
                break;
            }
            book.pin_module[static_cast<size_t>(first_pin + k)] = static_cast<int32_t>(module[k]);
        }
        if (mine.pin != kNoFailure) {
            const std::lock_guard<std::mutex> guard(failure_lock);
            if (mine.pin < failure.pin) failure = mine;
        }
    });

    // The first failure in file order: a repeated net name fails when its
    // header is read (PlacementDatabase::addNet), before the net's pins; a pin
    // fails at its line; an invalid header or the end of the file after every
    // pin read before it.
    const int64_t dup = net_table.firstDuplicate();
    const int64_t duplicate_key = dup < 0 ? std::numeric_limits<int64_t>::max() : 2 * book.net_pin_start[dup];
    const int64_t pin_key = failure.pin == std::numeric_limits<int64_t>::max() ? failure.pin : 2 * failure.pin + 1;
    const int64_t end_key = invalid_header >= 0 || truncated ? 2 * pins : std::numeric_limits<int64_t>::max();
    const int64_t key = std::min({duplicate_key, pin_key, end_key});
    if (key == std::numeric_limits<int64_t>::max()) return;
    if (key == duplicate_key) invalidArgument("Duplicate net name: " + std::string(net_names[dup]));
    if (key == pin_key) {
        // The last net starting at or before the pin holds it (empty nets end there).
        const size_t net = static_cast<size_t>(std::upper_bound(book.net_pin_start.begin(), book.net_pin_start.end(),
                                                                failure.pin) - book.net_pin_start.begin()) - 1;
        const int64_t rank = first_rank[net] + (failure.pin - book.net_pin_start[net]);
        if (!failure.unknown) parseError(path.string() + ": invalid pin at line " + std::to_string(lineNumber(rank)));
        parseError(path.string() + ": net '" + std::string(net_names[net]) + "' references unknown module '" +
                   std::string(failure.module) + "' at line " + std::to_string(lineNumber(rank)));
    }
    if (invalid_header >= 0) {
        parseError(path.string() + ": invalid NetDegree at line " + std::to_string(lineNumber(invalid_header)));
    }
    parseError(path.string() + ": unexpected end of file while reading net '" + std::string(net_names.back()) + "'");
}

// ---- .wts (BookshelfParser.cpp:265-278) -----------------------------------------------------

void parseWeights(Text text, const Workers& workers, const NameTable& nets, Bookshelf& book) {
    struct Records {
        std::vector<Text> names;
        std::vector<double> weight;
        std::vector<int64_t> net;
    };
    const std::vector<Piece> pieces = linePieces(text, workers.threads());
    std::vector<Records> parsed(pieces.size());
    workers.run(pieces.size(), [&](size_t i) {
        size_t pos = pieces[i].begin;
        while (pos < pieces[i].end) {
            const Text line = stripLine(nextLine(text, pos, pieces[i].end));
            if (line.empty() || beginsWith(line, "UCLA")) continue;
            Fields fields(line);
            Text name;
            double weight = 1.0;
            if (!(fields.word(name) && fields.real(weight))) continue;
            parsed[i].names.push_back(name);
            parsed[i].weight.push_back(weight);
        }
        parsed[i].net.resize(parsed[i].names.size());
        nets.findMany(parsed[i].names.data(), parsed[i].net.data(), parsed[i].names.size());
    });
    for (const Records& records : parsed) {
        for (size_t k = 0; k < records.net.size(); ++k) {
            if (records.net[k] >= 0) book.net_weight[static_cast<size_t>(records.net[k])] = records.weight[k];
        }
    }
}

}  // namespace

// BookshelfParser::parseAux (BookshelfParser.cpp:313-348): the files in the
// reference's order (.nodes, .scl, .pl, .nets, then .wts when named), then
// refreshDerivedData's terminal => fixed and validateCounts (:280-299).  The
// named files are read on their own threads while the earlier ones parse.
Bookshelf readBookshelf(const std::string& aux_name, int threads) {
    const Workers workers = threads > 0 ? Workers(threads) : Workers::all(kDefaultThreads);
    const fs::path aux_path(aux_name);
    const FileText aux = readWhole(aux_path);
    if (!aux.opened) parseError("Unable to open BookShelf file: " + aux_path.string());
    const std::unordered_map<std::string, fs::path> files = auxFiles(aux_path, aux.data);

    std::unordered_map<std::string, std::future<FileText>> reads;
    for (const char* extension : {".nodes", ".scl", ".pl", ".nets", ".wts"}) {
        const auto it = files.find(extension);
        if (it == files.end()) continue;
        std::error_code ignored;
        if (std::string(extension) == ".wts" && !fs::exists(it->second, ignored)) continue;
        reads.emplace(extension, std::async(std::launch::async, readWhole, it->second));
    }
    const auto required = [&](const std::string& extension) -> const fs::path& {
        const auto it = files.find(extension);
        if (it == files.end()) {
            parseError(aux_path.string() + ": missing required '" + extension + "' file in AUX record");
        }
        return it->second;
    };
    const auto contents = [&](const std::string& extension, const fs::path& path) {
        FileText file = reads.at(extension).get();
        if (!file.opened) parseError("Unable to open BookShelf file: " + path.string());
        return file;
    };

    Bookshelf book;
    std::optional<uint64_t> declared[4];
    std::vector<Text> module_names;
    NameTable module_table;
    const fs::path& nodes_path = required(".nodes");
    const FileText nodes = contents(".nodes", nodes_path);
    parseNodes(nodes_path, nodes.data, workers, book, module_names, module_table, declared);
    const fs::path& scl_path = required(".scl");
    parseScl(scl_path, contents(".scl", scl_path).data, book);
    const fs::path& pl_path = required(".pl");
    parsePl(pl_path, contents(".pl", pl_path).data, workers, module_table, book);
    const fs::path& nets_path = required(".nets");
    const FileText nets_file = contents(".nets", nets_path);
    std::vector<Text> net_names;
    NameTable net_table;
    parseNets(nets_path, nets_file.data, workers, module_table, book, net_names, net_table, declared + 2);
    book.net_weight.assign(net_names.size(), 1.0);
    if (const auto wts = files.find(".wts"); wts != files.end() && fs::exists(wts->second)) {
        const FileText weights = reads.count(".wts") != 0 ? contents(".wts", wts->second) : readWhole(wts->second);
        if (!weights.opened) parseError("Unable to open BookShelf file: " + wts->second.string());
        parseWeights(weights.data, workers, net_table, book);
    }

    // validateCounts (BookshelfParser.cpp:280-299).
    const auto check = [&](int k, const char* label, uint64_t actual) {
        if (declared[k] && *declared[k] != actual) {
            parseError(aux_path.string() + ": declared " + label + "=" + std::to_string(*declared[k]) + ", parsed " +
                       std::to_string(actual));
        }
    };
    uint64_t terminals = 0;
    for (const int32_t f : book.flags) terminals += (f & MPGP_MODULE_TERMINAL) != 0 ? 1 : 0;
    check(0, "NumNodes", module_names.size());
    check(1, "NumTerminals", terminals);
    check(2, "NumNets", net_names.size());
    check(3, "NumPins", book.pin_module.size());
    for (int k = 0; k < 4; ++k) book.declared[k] = declared[k] ? static_cast<int64_t>(*declared[k]) : -1;

    storeNames(module_names, workers, book.module_names, book.module_name_start);
    storeNames(net_names, workers, book.net_names, book.net_name_start);
    return book;
}

}  // namespace mpgp
