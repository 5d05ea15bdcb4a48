// TEST INFRASTRUCTURE ONLY.  The reference's per-step state output
// (new_dynamics.cpp:136-138, 233) lives in its main(), so its stream
// statement is restated here as a small program: it reads rows of six
// float64 (x, y, z, zeta, tracer, area) from argv[1] and appends
// "x,y,z,zeta,tracer,area" lines, default stream formatting, to argv[2].
#include <cstdio>
#include <fstream>
#include <vector>

using namespace std;

int main(int argc, char** argv) {
    if (argc != 3) return 2;
    FILE* in = fopen(argv[1], "rb");
    if (!in) return 3;
    vector<double> rows;
    double buf[6];
    while (fread(buf, sizeof(double), 6, in) == 6) rows.insert(rows.end(), buf, buf + 6);
    fclose(in);
    ofstream write_out1(argv[2], ofstream::out | ofstream::app);
    const size_t n = rows.size() / 6;
    for (size_t i = 0; i < n; i++) {
        const double* r = rows.data() + 6 * i;
        write_out1 << r[0] << "," << r[1] << "," << r[2] << "," << r[3] << "," << r[4] << "," << r[5] << "\n";
    }
    return write_out1.good() ? 0 : 1;
}
