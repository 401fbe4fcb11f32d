// Test driver for the reference's AllParams value parser (src/Util.cu, myatof),
// linked against the reference's own Util.cu object built by build_ref.sh:
// reads one token per line on stdin, prints the float's bits in hex.
#include <cstdint>
#include <cstdio>
#include <cstring>

float myatof(char s[]);

int main() {
    char buf[512];
    while (std::fgets(buf, sizeof(buf), stdin)) {
        buf[std::strcspn(buf, "\n")] = 0;
        float f = myatof(buf);
        uint32_t bits;
        std::memcpy(&bits, &f, 4);
        std::printf("%08x\n", bits);
    }
    return 0;
}
