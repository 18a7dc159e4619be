// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Decoder declarations (src/decode/block.rs, src/decode.rs).
#pragma once
#include <cstddef>
#include <cstdint>

#include "oracle_tables.h"

namespace oracle {

// Partition-set entry as the decoder tables hold it (block.rs:279-312 and
// :810-947): subset index of pixel `k` with 0x80 set on each subset's anchor
// pixel. Derived from the encoder tables (pattern + anchor "skip" table); a
// test checks the derivation against the decoder tables themselves.
inline uint32_t bptc_partition_set(uint32_t table_index, uint32_t k) {
    uint32_t subset = (kPatternTable[table_index] >> (2 * k)) & 3;
    uint32_t skip = kSkipTable[table_index];
    uint32_t anchor = subset == 0 ? 0 : (subset == 1 ? (skip >> 4) : (skip & 15));
    return subset | (k == anchor ? 0x80u : 0u);
}
inline uint32_t bc6h_partition_set(int32_t partition, int k) { return bptc_partition_set((uint32_t)partition, (uint32_t)k); }
inline uint32_t bc7_partition_set(uint32_t num_partitions, uint32_t partition, int k) {
    return bptc_partition_set(num_partitions == 3 ? 64 + partition : partition, (uint32_t)k);
}

void decode_block_bc1(const uint8_t* c, uint8_t* o, size_t pitch);
void decode_block_bc2(const uint8_t* c, uint8_t* o, size_t pitch);
void decode_block_bc3(const uint8_t* c, uint8_t* o, size_t pitch);
void decode_block_bc4(const uint8_t* c, uint8_t* o, size_t pitch);
void decode_block_bc5(const uint8_t* c, uint8_t* o, size_t pitch);
void decode_block_bc6h(const uint8_t* c, uint16_t* o, size_t pitch, bool is_signed);
void decode_block_bc6h_float(const uint8_t* c, float* o, size_t pitch, bool is_signed);
void decode_block_bc7(const uint8_t* c, uint8_t* o, size_t pitch);
uint8_t linear_to_srgb(float linear);
void decode_block_rgba8(int variant, const uint8_t* c, uint8_t* o, size_t pitch);

}  // namespace oracle
