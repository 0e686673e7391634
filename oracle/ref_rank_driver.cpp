// ref_rank_driver.cpp -- test infrastructure: runs the reference's own
// epic::BitVector (include/bit_vector.hpp:65-138) and epic::RankDataStructures
// (include/rank_data_structures.hpp:59-198), compiled from the reference's
// headers, on one bit-vector file and dumps what they compute:
//   u64 n_bits, u64 l0_words, u64 l12_words, u64 abs_ones, u64 padded_words,
//   then L0, L12 and the byte-swapped data words.
// Run it with MALLOC_PERTURB_=255 so that the bytes the reference leaves
// uninitialised in the last data word (bit_vector.hpp:119-124) read as zero.
#include <cstdio>
#include <cstdlib>

#include "include/rank_data_structures.hpp"

int main(int argc, char **argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: ref_rank <bitvector file> <bits_in_superblock> <kind 1|2> <out>\n");
        return 1;
    }
    const unsigned sb = (unsigned)std::atoi(argv[2]);
    const int kind = std::atoi(argv[3]);
    epic::BitVector bv;
    if (bv.create(argv[1])) return 2;
    if (bv.read()) return 3;
    epic::RankDataStructures rs;
    rs.create(sb, kind, bv);
    if (rs.construct(bv, 0ULL)) return 4;
    std::FILE *f = std::fopen(argv[4], "wb");
    if (!f) return 5;
    const unsigned long long hdr[5] = {bv.number_of_bits, rs.number_of_words_padded_layer_0,
                                       rs.number_of_words_padded_layer_12, rs.absolute_number_of_ones,
                                       bv.number_of_words_padded};
    std::fwrite(hdr, sizeof(hdr[0]), 5, f);
    std::fwrite(rs.layer_0, sizeof(u64), rs.number_of_words_padded_layer_0, f);
    std::fwrite(rs.layer_12, sizeof(u64), rs.number_of_words_padded_layer_12, f);
    std::fwrite(bv.data, sizeof(u64), bv.number_of_words_padded, f);
    std::fclose(f);
    return 0;
}
