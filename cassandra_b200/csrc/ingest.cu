// Training-data ingestion: the two on-disk forms of scored positions the
// reference reads, turned into the {P, O} uint64 records and scores that
// the fitting entry points take.
//
//  * binary records '<QQb' (NeuralNetwork/NeuralNetwork.py:21-29): player
//    and opponent bitboards as little-endian uint64, then the score as int8,
//    17 bytes per record, no header;
//  * text lines of ScoredPosition (Game/ScoredPosition.cpp:3-8 through
//    IO/File.cpp:16-24): Position::FromString (Board/Position.cpp:7-23) of
//    the line -- 64 board characters, 'X' a disc of the side in column 65,
//    'O' of the other, anything else empty, square i of the text is bit
//    63 - i -- then Score::FromString (Game/Score.cpp:6-15) of the text from
//    column 69: a sign character, decimal digits, halved toward zero, kept
//    as Score keeps it (int8, Game/Score.h).
//
// Host code; the records go to the device with one copy.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"

namespace cas {
namespace {

constexpr int64_t kRecordBytes = 17;

// Position::FromString of one line; false if the line is too short.
bool parse_position(const std::string& line, uint64_t& p, uint64_t& o)
{
    if (line.size() < 66) return false;
    uint64_t x = 0, y = 0;
    for (int i = 0; i < 64; i++) {
        if (line[i] == 'X')
            x |= uint64_t(1) << (63 - i);
        else if (line[i] == 'O')
            y |= uint64_t(1) << (63 - i);
    }
    if (line[65] == 'X') {
        p = x;
        o = y;
    } else {
        p = y;
        o = x;
    }
    return true;
}

// Score::FromString of the text from column 69: the digits after the first
// character (from_chars: stops at the first non-digit), negated if that
// character is '-', halved toward zero.  false if no digit follows.
bool parse_score(const std::string& line, int8_t& score)
{
    if (line.size() < 71) return false;
    int64_t v = 0;
    size_t i = 70;
    bool any = false;
    for (; i < line.size() && line[i] >= '0' && line[i] <= '9'; i++) {
        v = v * 10 + (line[i] - '0');
        any = true;
        if (v > 0x7fffffff) return false;
    }
    if (!any) return false;
    if (line[69] == '-') v = -v;
    score = static_cast<int8_t>(static_cast<int>(v / 2));
    return true;
}

}  // namespace
}  // namespace cas

using namespace cas;

extern "C" {

CAS_API cas_status cas_read_records(const char* path, uint64_t* h_positions, int8_t* h_scores, int64_t max_records,
                                    int64_t* n_records)
{
    CAS_REQUIRE(path && n_records && max_records >= 0, CAS_ERR_INVALID_ARGUMENT, "cas_read_records: bad argument");
    FILE* f = std::fopen(path, "rb");
    CAS_REQUIRE(f, CAS_ERR_INVALID_ARGUMENT, std::string("cas_read_records: cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const int64_t bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const int64_t n = bytes / kRecordBytes;  // a trailing partial record is not read, as the reference's loop stops
    if (!h_positions && !h_scores) {
        std::fclose(f);
        *n_records = n;
        return CAS_OK;
    }
    const int64_t take = n < max_records ? n : max_records;
    unsigned char rec[kRecordBytes];
    for (int64_t r = 0; r < take; r++) {
        if (std::fread(rec, 1, kRecordBytes, f) != static_cast<size_t>(kRecordBytes)) {
            std::fclose(f);
            set_error(std::string("cas_read_records: read failed: ") + path);
            return CAS_ERR_INVALID_ARGUMENT;
        }
        uint64_t p = 0, o = 0;
        for (int b = 7; b >= 0; b--) {
            p = (p << 8) | rec[b];
            o = (o << 8) | rec[8 + b];
        }
        if (h_positions) {
            h_positions[2 * r] = p;
            h_positions[2 * r + 1] = o;
        }
        if (h_scores) h_scores[r] = static_cast<int8_t>(rec[16]);
    }
    std::fclose(f);
    *n_records = take;
    return CAS_OK;
}

CAS_API cas_status cas_read_scored_positions(const char* path, uint64_t* h_positions, int8_t* h_scores,
                                             int64_t max_records, int64_t* n_records)
{
    CAS_REQUIRE(path && n_records && max_records >= 0, CAS_ERR_INVALID_ARGUMENT,
                "cas_read_scored_positions: bad argument");
    FILE* f = std::fopen(path, "rb");
    CAS_REQUIRE(f, CAS_ERR_INVALID_ARGUMENT, std::string("cas_read_scored_positions: cannot open ") + path);
    const bool count_only = !h_positions && !h_scores;
    int64_t n = 0, line_no = 0;
    std::string line;
    int c = 0;
    bool done = false;
    while (!done) {
        line.clear();
        while ((c = std::fgetc(f)) != EOF && c != '\n') line.push_back(static_cast<char>(c));
        done = c == EOF;
        if (done && line.empty()) break;  // no line after the last newline
        line_no++;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        uint64_t p = 0, o = 0;
        int8_t s = 0;
        if (!parse_position(line, p, o) || !parse_score(line, s)) {
            std::fclose(f);
            set_error("cas_read_scored_positions: line " + std::to_string(line_no) + " is not a scored position");
            return CAS_ERR_INVALID_ARGUMENT;
        }
        if (!count_only) {
            if (n >= max_records) break;
            if (h_positions) {
                h_positions[2 * n] = p;
                h_positions[2 * n + 1] = o;
            }
            if (h_scores) h_scores[n] = s;
        }
        n++;
    }
    std::fclose(f);
    *n_records = n;
    return CAS_OK;
}

}  // extern "C"
