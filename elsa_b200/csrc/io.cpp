// Image file formats (see io.hpp). Format rules follow io/EDFHandler.cpp:71-276,
// io/MHDHandler.cpp:68-218, io/PGMHandler.cpp:20-58 and io/ioUtils.cpp:10-123.
#include "io.hpp"

#include <algorithm>
#include <cctype>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <memory>
#include <sstream>

#include "internal.cuh"

namespace elsa_b200
{
    namespace io
    {
        namespace
        {
            [[noreturn]] void fail(const std::string& msg)
            {
                throw Error(ELSA_ERROR_INVALID_ARGUMENT, msg);
            }

            void trim(std::string& s)
            {
                s.erase(s.begin(), std::find_if(s.begin(), s.end(),
                                                [](int c) { return std::isspace(c) == 0; }));
                s.erase(std::find_if(s.rbegin(), s.rend(),
                                     [](int c) { return std::isspace(c) == 0; })
                            .base(),
                        s.end());
            }

            std::string lower(std::string s)
            {
                std::transform(s.begin(), s.end(), s.begin(),
                               [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
                return s;
            }

            std::string upper(std::string s)
            {
                std::transform(s.begin(), s.end(), s.begin(),
                               [](unsigned char c) { return static_cast<char>(std::toupper(c)); });
                return s;
            }

            // DataUtils::parse: one stream extraction that must not fail
            template <typename T>
            T parseOne(const std::string& str)
            {
                T v{};
                std::stringstream in(str);
                in >> v;
                if (in.fail())
                    fail("DataUtils::parse: failed to interpret string");
                return v;
            }

            // DataUtils::parseVector: extractions until the end of the string
            template <typename T>
            std::vector<T> parseList(const std::string& str)
            {
                std::vector<T> out;
                std::stringstream in(str);
                while (!in.eof()) {
                    T v{};
                    in >> v;
                    if (in.fail())
                        fail("DataUtils::parseVector: failed to interpret string");
                    out.push_back(v);
                }
                return out;
            }

            int64_t sizeOf(DataType t)
            {
                switch (t) {
                case DataType::INT8:
                case DataType::UINT8:
                    return 1;
                case DataType::INT16:
                case DataType::UINT16:
                    return 2;
                case DataType::INT32:
                case DataType::UINT32:
                case DataType::FLOAT32:
                    return 4;
                case DataType::FLOAT64:
                    return 8;
                }
                fail("DataUtils::getSizeOfDataType: unknown data type");
            }

            template <typename Raw>
            void convertRaw(std::istream& in, float* out, int64_t count)
            {
                const int64_t bytes = count * static_cast<int64_t>(sizeof(Raw));
                std::unique_ptr<Raw[]> tmp(new Raw[static_cast<size_t>(count)]);
                in.read(reinterpret_cast<char*>(tmp.get()), bytes);
                if (in.gcount() != bytes)
                    fail("DataUtils::parseRawData: failed to read sufficient data");
                for (int64_t i = 0; i < count; ++i)
                    out[i] = static_cast<float>(tmp[static_cast<size_t>(i)]);
            }

            // uint16, float32 and float64 raw data are readable (EDFHandler.cpp:30-37)
            void readRaw(std::istream& in, DataType t, float* out, int64_t count,
                         const char* who)
            {
                if (t == DataType::UINT16)
                    convertRaw<uint16_t>(in, out, count);
                else if (t == DataType::FLOAT32)
                    convertRaw<float>(in, out, count);
                else if (t == DataType::FLOAT64)
                    convertRaw<double>(in, out, count);
                else
                    fail(std::string(who) + ": invalid/unsupported data type");
            }

            // EDF::readHeader (EDFHandler.cpp:71-131): '{', then "name = value;" assignments
            // (';' inside quotes does not end one), names lower-cased, quotes stripped, up to '}'
            std::map<std::string, std::string> edfProperties(std::istream& file)
            {
                std::map<std::string, std::string> props;
                if (file.eof() || file.get() != '{')
                    fail("EDF::readHeader: no header opening marker");
                while (!file.eof()) {
                    while (!file.eof()) {
                        const int c = file.peek();
                        if (c != '\r' && c != '\n' && c != ' ' && c != '\t')
                            break;
                        file.ignore(1);
                    }
                    if (file.eof() || file.peek() == '}')
                        break;
                    bool q1 = false, q2 = false;
                    std::string assignment;
                    while (!file.eof()) {
                        const int got = file.get();
                        if (got == std::char_traits<char>::eof())
                            break;
                        const char c = static_cast<char>(got);
                        if (c == ';' && !(q1 || q2))
                            break;
                        if (c == '\'')
                            q1 = !q1;
                        if (c == '"')
                            q2 = !q2;
                        assignment += c;
                    }
                    const size_t eq = assignment.find('=');
                    if (eq == std::string::npos)
                        fail("failed reading name/value delimiter");
                    std::string name = assignment.substr(0, eq);
                    std::string value = assignment.substr(eq + 1);
                    trim(name);
                    trim(value);
                    if (!value.empty() && value.front() == value.back() &&
                        (value.front() == '\'' || value.front() == '"'))
                        value = value.size() >= 2 ? value.substr(1, value.size() - 2) : "";
                    props[lower(name)] = value;
                }
                file.ignore(2); // "}\n"
                return props;
            }

            // EDF::parseHeader (EDFHandler.cpp:133-216)
            ImageInfo edfParse(const std::map<std::string, std::string>& props)
            {
                ImageInfo info;
                for (int i = 1;; ++i) {
                    auto it = props.find("dim_" + std::to_string(i));
                    if (it == props.end())
                        break;
                    info.dims.push_back(parseOne<int64_t>(it->second));
                }
                if (info.dims.empty())
                    fail("EDF::parseHeader: dimension information not found");
                std::vector<float> spacing;
                if (auto it = props.find("spacing"); it != props.end())
                    spacing = parseList<float>(it->second);
                if (auto it = props.find("byteorder"); it != props.end())
                    if (lower(it->second) != "lowbytefirst")
                        fail("EDF::parseHeader: unsupported byte order value");
                auto dt = props.find("datatype");
                if (dt == props.end())
                    fail("EDF::parseHeader: data type not found");
                const std::string v = lower(dt->second);
                if (v == "signedbyte")
                    info.type = DataType::INT8;
                else if (v == "unsignedbyte")
                    info.type = DataType::UINT8;
                else if (v == "signedshort")
                    info.type = DataType::INT16;
                else if (v == "unsignedshort")
                    info.type = DataType::UINT16;
                else if (v == "float" || v == "floatvalue" || v == "real")
                    info.type = DataType::FLOAT32;
                else if (v == "double" || v == "doublevalue")
                    info.type = DataType::FLOAT64;
                else
                    fail("EDF::parseHeader: invalid/unsupported data type");
                if (props.count("compression"))
                    fail("EDF::parseHeader: compression not supported");
                int64_t size = 0;
                if (auto it = props.find("size"); it != props.end())
                    size = parseOne<int64_t>(it->second);
                if (auto it = props.find("image"); it != props.end())
                    if (parseOne<int64_t>(it->second) != 1)
                        fail("EDF::parseHeader: image not set to 1");
                if (info.count() * sizeOf(info.type) != size)
                    fail("EDF::parseHeader: size inconsistency");
                info.spacing.assign(info.dims.size(), 1.0f);
                if (!spacing.empty()) {
                    if (spacing.size() != info.dims.size())
                        fail("EDF::parseHeader: spacing inconsistency");
                    info.spacing = spacing;
                }
                return info;
            }

            // MHD::readHeader (MHDHandler.cpp:68-96): "name = value" lines, names lower-cased
            std::map<std::string, std::string> mhdProperties(std::istream& meta)
            {
                std::map<std::string, std::string> props;
                std::string line;
                while (std::getline(meta, line)) {
                    trim(line);
                    if (line.empty())
                        continue;
                    const size_t eq = line.find('=');
                    if (eq == std::string::npos)
                        fail("MHD::readHeader: found non-empty line without name/value pair");
                    std::string name = line.substr(0, eq);
                    std::string value = line.substr(eq + 1);
                    trim(name);
                    trim(value);
                    props[lower(name)] = value;
                }
                return props;
            }

            // MHD::parseHeader (MHDHandler.cpp:98-172); returns the data file name
            std::string mhdParse(const std::map<std::string, std::string>& props, ImageInfo& info)
            {
                auto nd = props.find("ndims");
                if (nd == props.end())
                    fail("MHD::parseHeader: tag 'ndims' not found");
                const int64_t nDims = parseOne<int64_t>(nd->second);
                if (auto it = props.find("elementbyteordermsb"); it != props.end()) {
                    const std::string v = lower(it->second);
                    if (v != "false" && v != "no")
                        fail("MHD::parseHeader: only supporting little endian byte order");
                }
                auto et = props.find("elementtype");
                if (et == props.end())
                    fail("MHD::parseHeader: tag 'element type' not found");
                const std::string v = upper(et->second);
                if (v == "MET_CHAR")
                    info.type = DataType::INT8;
                else if (v == "MET_UCHAR")
                    info.type = DataType::UINT8;
                else if (v == "MET_SHORT")
                    info.type = DataType::INT16;
                else if (v == "MET_USHORT")
                    info.type = DataType::UINT16;
                else if (v == "MET_FLOAT")
                    info.type = DataType::FLOAT32;
                else if (v == "MET_DOUBLE")
                    info.type = DataType::FLOAT64;
                else
                    fail("MHD::parseHeader: tag 'element type' of unsupported value");
                auto df = props.find("elementdatafile");
                if (df == props.end())
                    fail("MHD::parseHeader: tag 'element data file' not found");
                auto ds = props.find("dimsize");
                if (ds == props.end())
                    fail("MHD::parseHeader: tag 'dim size' not found");
                info.dims = parseList<int64_t>(ds->second);
                if (static_cast<int64_t>(info.dims.size()) != nDims)
                    fail("MHD::parseHeader: dimension size mismatch");
                info.spacing.assign(info.dims.size(), 1.0f);
                if (auto it = props.find("elementspacing"); it != props.end()) {
                    std::vector<float> sp = parseList<float>(it->second);
                    if (static_cast<int64_t>(sp.size()) != nDims)
                        fail("MHD::parseHeader: spacing size mismatch");
                    info.spacing = sp;
                }
                return df->second;
            }

            // FileSystemUtils::getAbsolutePath (ioUtils.cpp:104-123): relative to the meta
            // file's directory; an absolute data path is taken as it is
            std::string dataPath(const std::string& rel, const std::string& metaPath)
            {
                if (!rel.empty() && rel[0] == '/')
                    return rel;
                const size_t cut = metaPath.find_last_of("/\\");
                const std::string base = cut == std::string::npos ? "." : metaPath.substr(0, cut);
                char* resolved = realpath(base.c_str(), nullptr);
                if (!resolved)
                    fail("MHD::read: cannot resolve the directory of '" + metaPath + "'");
                std::string out(resolved);
                std::free(resolved);
                return out + "/" + rel;
            }

            // A vector as Eigen prints a transposed vector with the default IOFormat: every
            // coefficient right-aligned to the widest one, separated by one space.
            template <typename T>
            std::string eigenRow(const std::vector<T>& v)
            {
                size_t width = 0;
                std::vector<std::string> parts;
                for (const T& x : v) {
                    std::ostringstream s;
                    s << x;
                    parts.push_back(s.str());
                    width = std::max(width, parts.back().size());
                }
                std::ostringstream out;
                for (size_t i = 0; i < parts.size(); ++i) {
                    if (i)
                        out << ' ';
                    out << std::setw(static_cast<int>(width)) << parts[i];
                }
                return out.str();
            }

            void checkShape(const std::vector<int64_t>& dims, const std::vector<float>& spacing,
                            const char* who)
            {
                if (dims.empty())
                    fail(std::string(who) + ": no dimensions");
                for (int64_t d : dims)
                    if (d <= 0)
                        fail(std::string(who) + ": dimensions must be positive");
                if (spacing.size() != dims.size())
                    fail(std::string(who) + ": one spacing per dimension");
            }
        } // namespace

        int64_t ImageInfo::count() const
        {
            int64_t n = 1;
            for (int64_t d : dims)
                n *= d;
            return n;
        }

        ImageInfo edfInfo(const std::string& path)
        {
            std::ifstream file(path, std::ios::binary);
            if (!file.good())
                fail("EDF::read: cannot read from '" + path + "'");
            return edfParse(edfProperties(file));
        }

        void edfRead(const std::string& path, float* out, int64_t count)
        {
            std::ifstream file(path, std::ios::binary);
            if (!file.good())
                fail("EDF::read: cannot read from '" + path + "'");
            const ImageInfo info = edfParse(edfProperties(file));
            if (info.count() != count)
                fail("EDF::read: output buffer does not match the image size");
            readRaw(file, info.type, out, count, "EDF::read");
        }

        // EDF::writeHeader (EDFHandler.cpp:218-255): padded with spaces so that the header,
        // closed by "\n}\n", ends on a 1024-byte boundary
        std::string edfHeader(const std::vector<int64_t>& dims, const std::vector<float>& spacing)
        {
            checkShape(dims, spacing, "EDF::write");
            std::ostringstream h;
            h << "{\n";
            h << "HeaderID = EH:000001:000000:000000;\n";
            h << "Image = " << 1 << ";\n";
            h << "ByteOrder = LowByteFirst;\n";
            h << "DataType = FloatValue;\n";
            int64_t n = 1;
            for (size_t i = 0; i < dims.size(); ++i) {
                h << "Dim_" << (i + 1) << " = " << dims[i] << ";\n";
                n *= dims[i];
            }
            h << "Size = " << n * static_cast<int64_t>(sizeof(float)) << ";\n";
            h << "Spacing =";
            for (float s : spacing)
                h << ' ' << s;
            h << ";\n";
            const int64_t len = static_cast<int64_t>(h.str().size());
            int64_t padTo = 1024;
            while (padTo < len + 3)
                padTo += 1024;
            h << std::string(static_cast<size_t>(padTo - (len + 3)), ' ');
            h << "\n}\n";
            return h.str();
        }

        void edfWrite(const std::string& path, const float* data,
                      const std::vector<int64_t>& dims, const std::vector<float>& spacing)
        {
            const std::string header = edfHeader(dims, spacing);
            std::ofstream file(path, std::ios::binary);
            if (!file.good())
                fail("EDF::write: cannot write to '" + path + "'");
            file << header;
            int64_t n = 1;
            for (int64_t d : dims)
                n *= d;
            file.write(reinterpret_cast<const char*>(data),
                       static_cast<std::streamsize>(n * static_cast<int64_t>(sizeof(float))));
            if (!file.good())
                fail("EDF::write: write failed for '" + path + "'");
        }

        ImageInfo mhdInfo(const std::string& metaPath)
        {
            std::ifstream meta(metaPath);
            if (!meta.good())
                fail("MHD::read: cannot read from '" + metaPath + "'");
            ImageInfo info;
            mhdParse(mhdProperties(meta), info);
            return info;
        }

        void mhdRead(const std::string& metaPath, float* out, int64_t count)
        {
            std::ifstream meta(metaPath);
            if (!meta.good())
                fail("MHD::read: cannot read from '" + metaPath + "'");
            ImageInfo info;
            const std::string rel = mhdParse(mhdProperties(meta), info);
            if (info.count() != count)
                fail("MHD::read: output buffer does not match the image size");
            std::ifstream raw(dataPath(rel, metaPath), std::ios::binary | std::ios::in);
            if (!raw.good())
                fail("MHD::read: can not read from '" + rel + "'");
            readRaw(raw, info.type, out, count, "MHD::read");
        }

        // MHD::writeHeader (MHDHandler.cpp:174-194)
        std::string mhdHeader(const std::vector<int64_t>& dims, const std::vector<float>& spacing,
                              const std::string& rawPath)
        {
            checkShape(dims, spacing, "MHD::write");
            std::ostringstream h;
            h << "NDims = " << dims.size() << "\n";
            h << "DimSize = " << eigenRow(dims) << "\n";
            h << "ElementSpacing = " << eigenRow(spacing) << "\n";
            h << "ElementType = MET_FLOAT\n";
            h << "ElementByteOrderMSB = False\n";
            h << "ElementDataFile = " << rawPath << "\n";
            return h.str();
        }

        void mhdWrite(const std::string& metaPath, const std::string& rawPath, const float* data,
                      const std::vector<int64_t>& dims, const std::vector<float>& spacing)
        {
            const std::string header = mhdHeader(dims, spacing, rawPath);
            {
                std::ofstream meta(metaPath);
                if (!meta.good())
                    fail("MHD::write: cannot write to '" + metaPath + "'");
                meta << header;
            }
            std::ofstream raw(rawPath, std::ios::binary);
            if (!raw.good())
                fail("MHD::write: cannot write to '" + rawPath + "'");
            int64_t n = 1;
            for (int64_t d : dims)
                n *= d;
            raw.write(reinterpret_cast<const char*>(data),
                      static_cast<std::streamsize>(n * static_cast<int64_t>(sizeof(float))));
            if (!raw.good())
                fail("MHD::write: write failed for '" + rawPath + "'");
        }

        // PGM::write (PGMHandler.cpp:20-58): "P2", the two extents, 255, then every value as
        // int((v - min) * (255 / (max - min))), each followed by a space
        std::string pgmText(const float* data, const std::vector<int64_t>& dims)
        {
            const size_t d = dims.size();
            if (d != 2 && !(d == 3 && dims[2] == 1))
                fail("PGM:: Can only handle 2D data");
            int64_t n = 1;
            for (int64_t v : dims)
                n *= v;
            float mx = data[0], mn = data[0];
            for (int64_t i = 1; i < n; ++i) {
                mx = std::max(mx, data[i]);
                mn = std::min(mn, data[i]);
            }
            const float range = mx - mn;
            const float scale =
                range < std::numeric_limits<float>::epsilon() ? 0.0f : 255.0f / range;
            std::ostringstream out;
            out << "P2\n" << dims[0] << " " << dims[1] << "\n" << 255 << "\n";
            for (int64_t i = 0; i < n; ++i)
                out << static_cast<int>((data[i] - mn) * scale) << " ";
            return out.str();
        }

        void pgmWrite(const std::string& path, const float* data,
                      const std::vector<int64_t>& dims)
        {
            const std::string text = pgmText(data, dims);
            std::ofstream file(path, std::ios_base::out);
            if (!file.good())
                fail("PGM::write: cannot write to '" + path + "'");
            file << text;
        }
    } // namespace io
} // namespace elsa_b200
