// Min-max scalar quantizer (reference: nsparse/utils/scalar_quantizer.h:21-127),
// with the same float arithmetic, so codes and decoded scores match it bit
// for bit.
#ifndef NSPARSE_B200_SCALAR_QUANTIZER_H
#define NSPARSE_B200_SCALAR_QUANTIZER_H

#include <cstddef>
#include <cstdint>

namespace nsparse {

enum class QuantizerType : uint8_t {
    QT_8bit,
    QT_16bit,
};

class ScalarQuantizer {
public:
    ScalarQuantizer() : qtype_(QuantizerType::QT_8bit), vmin_(0), vmax_(1) {}
    // Throws std::invalid_argument for a non-finite or empty range.
    ScalarQuantizer(QuantizerType qtype, float vmin, float vmax);

    size_t bytes_per_value() const { return qtype_ == QuantizerType::QT_8bit ? 1 : 2; }
    int bits() const { return qtype_ == QuantizerType::QT_8bit ? 8 : 16; }
    void encode(const float* vals, uint8_t* codes, size_t n) const;
    void decode(const uint8_t* codes, float* vals, size_t n) const;
    QuantizerType get_quantizer_type() const { return qtype_; }
    float get_min() const { return vmin_; }
    float get_max() const { return vmax_; }
    // kMax / (vmax - vmin), the factor encode applies after subtracting vmin.
    float encode_scale() const;
    // The factor decode_dot_product multiplies a quantized score by.
    float decode_scale(const ScalarQuantizer& query_sq) const;
    float decode_dot_product(float quantized_score, const ScalarQuantizer& query_sq) const {
        return quantized_score * decode_scale(query_sq);
    }

private:
    QuantizerType qtype_;
    float vmin_;
    float vmax_;
};

}  // namespace nsparse

#endif
