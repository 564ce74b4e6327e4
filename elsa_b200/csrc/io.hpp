// Image file formats of elsa's io module (io/EDFHandler.cpp, io/MHDHandler.cpp,
// io/PGMHandler.cpp, io/ioUtils.cpp) on host buffers of float: headers are written byte for byte
// as the reference writes them and parsed with the reference's rules and error cases.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace elsa_b200
{
    namespace io
    {
        // element types of the raw data (DataUtils::DataType, io/ioUtils.h:33-45)
        enum class DataType { INT8, UINT8, INT16, UINT16, INT32, UINT32, FLOAT32, FLOAT64 };

        struct ImageInfo {
            std::vector<int64_t> dims;  // coefficients per dimension (x first)
            std::vector<float> spacing; // per dimension (1 when the file gives none)
            DataType type = DataType::FLOAT32;
            int64_t count() const;
        };

        // EDF: header and raw little-endian data in one file.
        ImageInfo edfInfo(const std::string& path);
        // reads edfInfo(path).count() values, converted to float, into out
        void edfRead(const std::string& path, float* out, int64_t count);
        std::string edfHeader(const std::vector<int64_t>& dims, const std::vector<float>& spacing);
        void edfWrite(const std::string& path, const float* data,
                      const std::vector<int64_t>& dims, const std::vector<float>& spacing);

        // MHD: a text meta file naming a raw data file (relative names resolve against the
        // meta file's directory).
        ImageInfo mhdInfo(const std::string& metaPath);
        void mhdRead(const std::string& metaPath, float* out, int64_t count);
        std::string mhdHeader(const std::vector<int64_t>& dims, const std::vector<float>& spacing,
                              const std::string& rawPath);
        void mhdWrite(const std::string& metaPath, const std::string& rawPath, const float* data,
                      const std::vector<int64_t>& dims, const std::vector<float>& spacing);

        // PGM (P2 grey scale, values scaled to [0, 255]) of 2D data, or 3D data with a last
        // dimension of 1.
        std::string pgmText(const float* data, const std::vector<int64_t>& dims);
        void pgmWrite(const std::string& path, const float* data,
                      const std::vector<int64_t>& dims);
    } // namespace io
} // namespace elsa_b200
