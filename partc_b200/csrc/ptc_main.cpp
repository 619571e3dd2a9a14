// Drop-in driver with the reference's command line and stdout lines (main.cpp:29-191):
//
//     ptc_tc <tensor.tns> <tensor.meta> <isMtx 0/1> <numTests>
//
// It reads the tensor (FROSTT text, 1-based, on the GPU with ptc_read_tns, which gives what
// readTensor in mtxTnsIO.cpp:30-65 gives; or a MatrixMarket coordinate file on the host when isMtx
// is 1, like readMatrix), reads the meta file like
// Tensor::populate_meta_info (tensor.hpp:151-173), prints the mode sizes like main.cpp:107-109,
// and replaces main.cpp:112-118 (B = A, both hash tables, tc_fksCuckoo) with one call to
// ptc_self_contract.  The library prints the reference's timing and nnz lines.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "partc.h"

namespace {

bool read_mtx(const std::string& path, std::vector<uint32_t>& idx, std::vector<double>& vals,
              std::vector<uint32_t>& dims, uint32_t& d) {
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    bool header = false;
    d = 2;
    dims.assign(2, 0);
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '%') continue;
        std::istringstream ls(line);
        if (!header) {  // rows cols nnz
            header = true;
            continue;
        }
        uint64_t i = 0, j = 0;
        double v = 1.0;
        ls >> i >> j;
        if (!(ls >> v)) v = 1.0;
        idx.push_back((uint32_t)(i - 1));
        idx.push_back((uint32_t)(j - 1));
        vals.push_back(v);
        if (i > dims[0]) dims[0] = (uint32_t)i;
        if (j > dims[1]) dims[1] = (uint32_t)j;
    }
    return header;
}

bool read_meta(const std::string& path, uint32_t d, uint32_t& c, std::vector<uint32_t>& dim_tc) {
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    for (int i = 0; i < 2; ++i) std::getline(in, line);  // two comment lines
    if (!(in >> c)) return false;
    dim_tc.resize(d);
    for (uint32_t i = 0; i < d; ++i)
        if (!(in >> dim_tc[i])) return false;
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "input not parsed correctly!\n" << std::endl;
        std::cerr << "Usage : \n\t" << argv[0] << "\n"
                  << "\tfilename tensor A   : tensor A\n"
                  << "\tfilename tensor A meta info : contraction specific info for tensor A\n"
                  << "\tisMtx : 0 => tensor; 1 => matrix\n"
                  << "\tnumber of rounds : number of times to run the experiment\n";
        return 1;
    }
    const std::string file_a = argv[1], file_meta = argv[2];
    const int is_mtx = atoi(argv[3]);
    std::vector<uint32_t> idx, dims, dim_tc;
    std::vector<double> vals;
    uint32_t d = 0, c = 0;
    ptc_tensor dev_in;  // a .tns file is read on the GPU and stays there
    std::memset(&dev_in, 0, sizeof(dev_in));
    bool ok = false;
    if (is_mtx) {
        ok = read_mtx(file_a, idx, vals, dims, d);
    } else {
        ptc_options ro;
        ptc_options_init(&ro);
        ro.output_location = PTC_DEVICE;
        uint32_t dm[16];
        ok = ptc_read_tns(file_a.c_str(), &ro, &dev_in, dm) == PTC_OK;
        if (ok) {
            d = dev_in.order;
            dims.assign(dm, dm + d);
        } else {
            std::cerr << ptc_last_error() << std::endl;
        }
    }
    if (!ok) {
        std::cerr << "Could not read \"" << file_a << "\"" << std::endl;
        return 1;
    }
    if (!read_meta(file_meta, d, c, dim_tc)) {
        std::cerr << "Could not open the file \"" << file_meta << "\"" << std::endl;
        return 1;
    }
    for (uint32_t j = 0; j < d; ++j) std::cout << dims[j] << " \n"[j + 1 == d];
    std::cout << std::flush;

    ptc_options opt;
    ptc_options_init(&opt);
    opt.verbose = 1;
    ptc_tensor out;
    ptc_stats stats;
    ptc_status s;
    if (is_mtx) {
        s = ptc_self_contract(idx.data(), vals.data(), d, vals.size(), dims.data(), c, dim_tc.data(), &opt, &out,
                              &stats);
    } else {
        ptc_coo A;
        A.order = d;
        A.location = PTC_DEVICE;
        A.nnz = dev_in.nnz;
        A.idx = dev_in.idx;
        A.vals = dev_in.vals;
        A.dims = dims.data();
        // the reference's self-contraction rule: B = A needs more than one nonzero
        s = A.nnz > 1 ? ptc_contract(&A, nullptr, c, dim_tc.data(), dim_tc.data(), &opt, &out, &stats)
                      : PTC_ERR_TOO_FEW_NONZEROS;
        ptc_tensor_free(&dev_in);
    }
    if (s != PTC_OK) {
        std::cerr << ptc_status_string(s) << ": " << ptc_last_error() << std::endl;
        return 1;
    }
    ptc_tensor_free(&out);
    return 0;
}
