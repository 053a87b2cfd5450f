// GENERATED by warpsphboundaries_b200/kernels.py (emit_header); do not edit by hand.
// Exact rational kernel profiles rounded once to double; see that module for the algebra.
#pragma once

namespace wsb {

constexpr int kNumKernels = 10;
constexpr int kMaxA = 14;   // A_n, n = 0 .. kMaxA-1

struct BlockSums {      // per (pair, block) chord sums, before the 1/pi and the edge frame
  double W0, W1;        // int P ds, int s P ds
  double P0, P1;        // int Psi ds, int s Psi ds
  double Lreg, Preg;    // int M/r^2 ds, int MPsi/r^2 ds (regular parts of the value terms)
  double Mhat, MPhat;   // singular coefficients M(R), MPsi(R)
};

struct AdjSums {        // per (pair, block) chord sums of the adjoint
  double W0, W1, W2, W3;   // int s^j P ds, j = 0..3
};

// ---- cubic: C2*pi = 80/7, plane second moment 31/392
struct Kern_cubic {
  static constexpr int kId = 0;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 2;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.07908163265306123;
  static constexpr double kR[kBlocks] = {1.0, 0.5};
  static constexpr int kNA[kBlocks] = {6, 6};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {6, 6};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_cubic::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['80/7', '-240/7', '240/7', '-80/7']
  o.W0 = 11.428571428571429*A[0] + -34.285714285714285*A[1] + 34.285714285714285*A[2] + -11.428571428571429*A[3];
  o.W1 = (((fma(fma(fma(-2.2857142857142856, rhi, 8.571428571428571), rhi, -11.428571428571429), rhi, 5.714285714285714))*rhi)*rhi) - (((fma(fma(fma(-2.2857142857142856, rlo, 8.571428571428571), rlo, -11.428571428571429), rlo, 5.714285714285714))*rlo)*rlo);
  o.P0 = -0.5714285714285714*A[0] + 5.714285714285714*A[2] + -11.428571428571429*A[3] + 8.571428571428571*A[4] + -2.2857142857142856*A[5];
  o.P1 = (((fma(fma(fma(fma(fma(-0.32653061224489793, rhi, 1.4285714285714286), rhi, -2.2857142857142856), rhi, 1.4285714285714286), rhi, 0.0), rhi, -0.2857142857142857))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-0.32653061224489793, rlo, 1.4285714285714286), rlo, -2.2857142857142856), rlo, 1.4285714285714286), rlo, 0.0), rlo, -0.2857142857142857))*rlo)*rlo);
  o.Lreg = 5.714285714285714*A[0] + -11.428571428571429*A[1] + 8.571428571428571*A[2] + -2.2857142857142856*A[3];
  o.Preg = -0.2857142857142857*A[0] + 1.4285714285714286*A[2] + -2.2857142857142856*A[3] + 1.4285714285714286*A[4] + -0.32653061224489793*A[5];
  o.Mhat = 0.5714285714285714;
  o.MPhat = -0.04081632653061224;
}
template <> __host__ __device__ __forceinline__ void Kern_cubic::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 11.428571428571429*A[0] + -34.285714285714285*A[1] + 34.285714285714285*A[2] + -11.428571428571429*A[3];
  const double a2 = 11.428571428571429*A[2] + -34.285714285714285*A[3] + 34.285714285714285*A[4] + -11.428571428571429*A[5];
  const double m1 = (((fma(fma(fma(-2.2857142857142856, rhi, 8.571428571428571), rhi, -11.428571428571429), rhi, 5.714285714285714))*rhi)*rhi) - (((fma(fma(fma(-2.2857142857142856, rlo, 8.571428571428571), rlo, -11.428571428571429), rlo, 5.714285714285714))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(-1.6326530612244898, rhi, 5.714285714285714), rhi, -6.857142857142857), rhi, 2.857142857142857))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(-1.6326530612244898, rlo, 5.714285714285714), rlo, -6.857142857142857), rlo, 2.857142857142857))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}
template <> __host__ __device__ __forceinline__ void Kern_cubic::sums<1>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1/2: P = ['-40/7', '240/7', '-480/7', '320/7']
  o.W0 = -5.714285714285714*A[0] + 34.285714285714285*A[1] + -68.57142857142857*A[2] + 45.714285714285715*A[3];
  o.W1 = (((fma(fma(fma(9.142857142857142, rhi, -17.142857142857142), rhi, 11.428571428571429), rhi, -2.857142857142857))*rhi)*rhi) - (((fma(fma(fma(9.142857142857142, rlo, -17.142857142857142), rlo, 11.428571428571429), rlo, -2.857142857142857))*rlo)*rlo);
  o.P0 = 0.07142857142857142*A[0] + -2.857142857142857*A[2] + 11.428571428571429*A[3] + -17.142857142857142*A[4] + 9.142857142857142*A[5];
  o.P1 = (((fma(fma(fma(fma(fma(1.3061224489795917, rhi, -2.857142857142857), rhi, 2.2857142857142856), rhi, -0.7142857142857143), rhi, 0.0), rhi, 0.03571428571428571))*rhi)*rhi) - (((fma(fma(fma(fma(fma(1.3061224489795917, rlo, -2.857142857142857), rlo, 2.2857142857142856), rlo, -0.7142857142857143), rlo, 0.0), rlo, 0.03571428571428571))*rlo)*rlo);
  o.Lreg = -2.857142857142857*A[0] + 11.428571428571429*A[1] + -17.142857142857142*A[2] + 9.142857142857142*A[3];
  o.Preg = 0.03571428571428571*A[0] + -0.7142857142857143*A[2] + 2.2857142857142856*A[3] + -2.857142857142857*A[4] + 1.3061224489795917*A[5];
  o.Mhat = -0.07142857142857142;
  o.MPhat = 0.0012755102040816326;
}
template <> __host__ __device__ __forceinline__ void Kern_cubic::adj<1>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = -5.714285714285714*A[0] + 34.285714285714285*A[1] + -68.57142857142857*A[2] + 45.714285714285715*A[3];
  const double a2 = -5.714285714285714*A[2] + 34.285714285714285*A[3] + -68.57142857142857*A[4] + 45.714285714285715*A[5];
  const double m1 = (((fma(fma(fma(9.142857142857142, rhi, -17.142857142857142), rhi, 11.428571428571429), rhi, -2.857142857142857))*rhi)*rhi) - (((fma(fma(fma(9.142857142857142, rlo, -17.142857142857142), rlo, 11.428571428571429), rlo, -2.857142857142857))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(6.530612244897959, rhi, -11.428571428571429), rhi, 6.857142857142857), rhi, -1.4285714285714286))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(6.530612244897959, rlo, -11.428571428571429), rlo, 6.857142857142857), rlo, -1.4285714285714286))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- w2: C2*pi = 7, plane second moment 5/72
struct Kern_w2 {
  static constexpr int kId = 1;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.06944444444444445;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {8};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {8};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_w2::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['7', '0', '-70', '140', '-105', '28']
  o.W0 = 7.0*A[0] + -70.0*A[2] + 140.0*A[3] + -105.0*A[4] + 28.0*A[5];
  o.W1 = (((fma(fma(fma(fma(fma(4.0, rhi, -17.5), rhi, 28.0), rhi, -17.5), rhi, 0.0), rhi, 3.5))*rhi)*rhi) - (((fma(fma(fma(fma(fma(4.0, rlo, -17.5), rlo, 28.0), rlo, -17.5), rlo, 0.0), rlo, 3.5))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 3.5*A[2] + -17.5*A[4] + 28.0*A[5] + -17.5*A[6] + 4.0*A[7];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(0.4444444444444444, rhi, -2.1875), rhi, 4.0), rhi, -2.9166666666666665), rhi, 0.0), rhi, 0.875), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(0.4444444444444444, rlo, -2.1875), rlo, 4.0), rlo, -2.9166666666666665), rlo, 0.0), rlo, 0.875), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 3.5*A[0] + -17.5*A[2] + 28.0*A[3] + -17.5*A[4] + 4.0*A[5];
  o.Preg = -0.25*A[0] + 0.875*A[2] + -2.9166666666666665*A[4] + 4.0*A[5] + -2.1875*A[6] + 0.4444444444444444*A[7];
  o.Mhat = 0.5;
  o.MPhat = -0.034722222222222224;
}
template <> __host__ __device__ __forceinline__ void Kern_w2::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 7.0*A[0] + -70.0*A[2] + 140.0*A[3] + -105.0*A[4] + 28.0*A[5];
  const double a2 = 7.0*A[2] + -70.0*A[4] + 140.0*A[5] + -105.0*A[6] + 28.0*A[7];
  const double m1 = (((fma(fma(fma(fma(fma(4.0, rhi, -17.5), rhi, 28.0), rhi, -17.5), rhi, 0.0), rhi, 3.5))*rhi)*rhi) - (((fma(fma(fma(fma(fma(4.0, rlo, -17.5), rlo, 28.0), rlo, -17.5), rlo, 0.0), rlo, 3.5))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(3.111111111111111, rhi, -13.125), rhi, 20.0), rhi, -11.666666666666666), rhi, 0.0), rhi, 1.75))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(3.111111111111111, rlo, -13.125), rlo, 20.0), rlo, -11.666666666666666), rlo, 0.0), rlo, 1.75))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- w4: C2*pi = 9, plane second moment 7/132
struct Kern_w4 {
  static constexpr int kId = 2;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.05303030303030303;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {11};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {11};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_w4::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['9', '0', '-84', '0', '630', '-1344', '1260', '-576', '105']
  o.W0 = 9.0*A[0] + -84.0*A[2] + 630.0*A[4] + -1344.0*A[5] + 1260.0*A[6] + -576.0*A[7] + 105.0*A[8];
  o.W1 = (((fma(fma(fma(fma(fma(fma(fma(fma(10.5, rhi, -64.0), rhi, 157.5), rhi, -192.0), rhi, 105.0), rhi, 0.0), rhi, -21.0), rhi, 0.0), rhi, 4.5))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(10.5, rlo, -64.0), rlo, 157.5), rlo, -192.0), rlo, 105.0), rlo, 0.0), rlo, -21.0), rlo, 0.0), rlo, 4.5))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 4.5*A[2] + -21.0*A[4] + 105.0*A[6] + -192.0*A[7] + 157.5*A[8] + -64.0*A[9] + 10.5*A[10];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(0.875, rhi, -5.818181818181818), rhi, 15.75), rhi, -21.333333333333332), rhi, 13.125), rhi, 0.0), rhi, -3.5), rhi, 0.0), rhi, 1.125), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(0.875, rlo, -5.818181818181818), rlo, 15.75), rlo, -21.333333333333332), rlo, 13.125), rlo, 0.0), rlo, -3.5), rlo, 0.0), rlo, 1.125), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 4.5*A[0] + -21.0*A[2] + 105.0*A[4] + -192.0*A[5] + 157.5*A[6] + -64.0*A[7] + 10.5*A[8];
  o.Preg = -0.25*A[0] + 1.125*A[2] + -3.5*A[4] + 13.125*A[6] + -21.333333333333332*A[7] + 15.75*A[8] + -5.818181818181818*A[9] + 0.875*A[10];
  o.Mhat = 0.5;
  o.MPhat = -0.026515151515151516;
}
template <> __host__ __device__ __forceinline__ void Kern_w4::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 9.0*A[0] + -84.0*A[2] + 630.0*A[4] + -1344.0*A[5] + 1260.0*A[6] + -576.0*A[7] + 105.0*A[8];
  const double a2 = 9.0*A[2] + -84.0*A[4] + 630.0*A[6] + -1344.0*A[7] + 1260.0*A[8] + -576.0*A[9] + 105.0*A[10];
  const double m1 = (((fma(fma(fma(fma(fma(fma(fma(fma(10.5, rhi, -64.0), rhi, 157.5), rhi, -192.0), rhi, 105.0), rhi, 0.0), rhi, -21.0), rhi, 0.0), rhi, 4.5))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(10.5, rlo, -64.0), rlo, 157.5), rlo, -192.0), rlo, 105.0), rlo, 0.0), rlo, -21.0), rlo, 0.0), rlo, 4.5))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(fma(fma(fma(8.75, rhi, -52.36363636363637), rhi, 126.0), rhi, -149.33333333333334), rhi, 78.75), rhi, 0.0), rhi, -14.0), rhi, 0.0), rhi, 2.25))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(fma(fma(fma(8.75, rlo, -52.36363636363637), rlo, 126.0), rlo, -149.33333333333334), rlo, 78.75), rlo, 0.0), rlo, -14.0), rlo, 0.0), rlo, 2.25))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- w6: C2*pi = 78/7, plane second moment 3/70
struct Kern_w6 {
  static constexpr int kId = 3;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.04285714285714286;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {14};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {14};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_w6::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['78/7', '0', '-858/7', '0', '5148/7', '0', '-5148', '82368/7', '-12870', '54912/7', '-2574', '2496/7']
  o.W0 = 11.142857142857142*A[0] + -122.57142857142857*A[2] + 735.4285714285714*A[4] + -5148.0*A[6] + 11766.857142857143*A[7] + -12870.0*A[8] + 7844.571428571428*A[9] + -2574.0*A[10] + 356.57142857142856*A[11];
  o.W1 = (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(27.428571428571427, rhi, -214.5), rhi, 713.1428571428571), rhi, -1287.0), rhi, 1307.4285714285713), rhi, -643.5), rhi, 0.0), rhi, 122.57142857142857), rhi, 0.0), rhi, -30.642857142857142), rhi, 0.0), rhi, 5.571428571428571))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(27.428571428571427, rlo, -214.5), rlo, 713.1428571428571), rlo, -1287.0), rlo, 1307.4285714285713), rlo, -643.5), rlo, 0.0), rlo, 122.57142857142857), rlo, 0.0), rlo, -30.642857142857142), rlo, 0.0), rlo, 5.571428571428571))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 5.571428571428571*A[2] + -30.642857142857142*A[4] + 122.57142857142857*A[6] + -643.5*A[8] + 1307.4285714285713*A[9] + -1287.0*A[10] + 713.1428571428571*A[11] + -214.5*A[12] + 27.428571428571427*A[13];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.8285714285714285, rhi, -15.321428571428571), rhi, 54.857142857142854), rhi, -107.25), rhi, 118.85714285714286), rhi, -64.35), rhi, 0.0), rhi, 15.321428571428571), rhi, 0.0), rhi, -5.107142857142857), rhi, 0.0), rhi, 1.3928571428571428), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.8285714285714285, rlo, -15.321428571428571), rlo, 54.857142857142854), rlo, -107.25), rlo, 118.85714285714286), rlo, -64.35), rlo, 0.0), rlo, 15.321428571428571), rlo, 0.0), rlo, -5.107142857142857), rlo, 0.0), rlo, 1.3928571428571428), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 5.571428571428571*A[0] + -30.642857142857142*A[2] + 122.57142857142857*A[4] + -643.5*A[6] + 1307.4285714285713*A[7] + -1287.0*A[8] + 713.1428571428571*A[9] + -214.5*A[10] + 27.428571428571427*A[11];
  o.Preg = -0.25*A[0] + 1.3928571428571428*A[2] + -5.107142857142857*A[4] + 15.321428571428571*A[6] + -64.35*A[8] + 118.85714285714286*A[9] + -107.25*A[10] + 54.857142857142854*A[11] + -15.321428571428571*A[12] + 1.8285714285714285*A[13];
  o.Mhat = 0.5;
  o.MPhat = -0.02142857142857143;
}
template <> __host__ __device__ __forceinline__ void Kern_w6::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 11.142857142857142*A[0] + -122.57142857142857*A[2] + 735.4285714285714*A[4] + -5148.0*A[6] + 11766.857142857143*A[7] + -12870.0*A[8] + 7844.571428571428*A[9] + -2574.0*A[10] + 356.57142857142856*A[11];
  const double a2 = 11.142857142857142*A[2] + -122.57142857142857*A[4] + 735.4285714285714*A[6] + -5148.0*A[8] + 11766.857142857143*A[9] + -12870.0*A[10] + 7844.571428571428*A[11] + -2574.0*A[12] + 356.57142857142856*A[13];
  const double m1 = (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(27.428571428571427, rhi, -214.5), rhi, 713.1428571428571), rhi, -1287.0), rhi, 1307.4285714285713), rhi, -643.5), rhi, 0.0), rhi, 122.57142857142857), rhi, 0.0), rhi, -30.642857142857142), rhi, 0.0), rhi, 5.571428571428571))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(27.428571428571427, rlo, -214.5), rlo, 713.1428571428571), rlo, -1287.0), rlo, 1307.4285714285713), rlo, -643.5), rlo, 0.0), rlo, 122.57142857142857), rlo, 0.0), rlo, -30.642857142857142), rlo, 0.0), rlo, 5.571428571428571))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(23.771428571428572, rhi, -183.85714285714286), rhi, 603.4285714285714), rhi, -1072.5), rhi, 1069.7142857142858), rhi, -514.8), rhi, 0.0), rhi, 91.92857142857143), rhi, 0.0), rhi, -20.428571428571427), rhi, 0.0), rhi, 2.7857142857142856))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(23.771428571428572, rlo, -183.85714285714286), rlo, 603.4285714285714), rlo, -1072.5), rlo, 1069.7142857142858), rlo, -514.8), rlo, 0.0), rlo, 91.92857142857143), rlo, 0.0), rlo, -20.428571428571427), rlo, 0.0), rlo, 2.7857142857142856))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- quartic: C2*pi = 46875/2398, plane second moment 9759/152600
struct Kern_quartic {
  static constexpr int kId = 4;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 3;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.06395150720838794;
  static constexpr double kR[kBlocks] = {1.0, 0.6, 0.2};
  static constexpr int kNA[kBlocks] = {7, 7, 7};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {7, 7, 7};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_quartic::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['46875/2398', '-93750/1199', '140625/1199', '-93750/1199', '46875/2398']
  o.W0 = 19.547539616346956*A[0] + -78.19015846538782*A[1] + 117.28523769808173*A[2] + -78.19015846538782*A[3] + 19.547539616346956*A[4];
  o.W1 = (((fma(fma(fma(fma(3.2579232693911595, rhi, -15.638031693077565), rhi, 29.321309424520432), rhi, -26.063386155129276), rhi, 9.773769808173478))*rhi)*rhi) - (((fma(fma(fma(fma(3.2579232693911595, rlo, -15.638031693077565), rlo, 29.321309424520432), rlo, -26.063386155129276), rlo, 9.773769808173478))*rlo)*rlo);
  o.P0 = -0.6515846538782318*A[0] + 9.773769808173478*A[2] + -26.063386155129276*A[3] + 29.321309424520432*A[4] + -15.638031693077565*A[5] + 3.2579232693911595*A[6];
  o.P1 = (((fma(fma(fma(fma(fma(fma(0.40724040867389494, rhi, -2.2340045275825093), rhi, 4.886884904086739), rhi, -5.212677231025855), rhi, 2.4434424520433695), rhi, 0.0), rhi, -0.3257923269391159))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(0.40724040867389494, rlo, -2.2340045275825093), rlo, 4.886884904086739), rlo, -5.212677231025855), rlo, 2.4434424520433695), rlo, 0.0), rlo, -0.3257923269391159))*rlo)*rlo);
  o.Lreg = 9.773769808173478*A[0] + -26.063386155129276*A[1] + 29.321309424520432*A[2] + -15.638031693077565*A[3] + 3.2579232693911595*A[4];
  o.Preg = -0.3257923269391159*A[0] + 2.4434424520433695*A[2] + -5.212677231025855*A[3] + 4.886884904086739*A[4] + -2.2340045275825093*A[5] + 0.40724040867389494*A[6];
  o.Mhat = 0.6515846538782318;
  o.MPhat = -0.03490632074347671;
}
template <> __host__ __device__ __forceinline__ void Kern_quartic::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 19.547539616346956*A[0] + -78.19015846538782*A[1] + 117.28523769808173*A[2] + -78.19015846538782*A[3] + 19.547539616346956*A[4];
  const double a2 = 19.547539616346956*A[2] + -78.19015846538782*A[3] + 117.28523769808173*A[4] + -78.19015846538782*A[5] + 19.547539616346956*A[6];
  const double m1 = (((fma(fma(fma(fma(3.2579232693911595, rhi, -15.638031693077565), rhi, 29.321309424520432), rhi, -26.063386155129276), rhi, 9.773769808173478))*rhi)*rhi) - (((fma(fma(fma(fma(3.2579232693911595, rlo, -15.638031693077565), rlo, 29.321309424520432), rlo, -26.063386155129276), rlo, 9.773769808173478))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(2.4434424520433695, rhi, -11.170022637912545), rhi, 19.547539616346956), rhi, -15.638031693077565), rhi, 4.886884904086739))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(2.4434424520433695, rlo, -11.170022637912545), rlo, 19.547539616346956), rlo, -15.638031693077565), rlo, 4.886884904086739))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}
template <> __host__ __device__ __forceinline__ void Kern_quartic::sums<1>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 3/5: P = ['-30375/2398', '101250/1199', '-253125/1199', '281250/1199', '-234375/2398']
  o.W0 = -12.666805671392828*A[0] + 84.44537114261885*A[1] + -211.11342785654713*A[2] + 234.57047539616346*A[3] + -97.73769808173478*A[4];
  o.W1 = (((fma(fma(fma(fma(-16.289616346955796, rhi, 46.914095079232695), rhi, -52.77835696413678), rhi, 28.148457047539615), rhi, -6.333402835696414))*rhi)*rhi) - (((fma(fma(fma(fma(-16.289616346955796, rlo, 46.914095079232695), rlo, -52.77835696413678), rlo, 28.148457047539615), rlo, -6.333402835696414))*rlo)*rlo);
  o.P0 = 0.15200166805671392*A[0] + -6.333402835696414*A[2] + 28.148457047539615*A[3] + -52.77835696413678*A[4] + 46.914095079232695*A[5] + -16.289616346955796*A[6];
  o.P1 = (((fma(fma(fma(fma(fma(fma(-2.0362020433694745, rhi, 6.702013582747528), rhi, -8.79639282735613), rhi, 5.629691409507923), rhi, -1.5833507089241035), rhi, 0.0), rhi, 0.07600083402835696))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(-2.0362020433694745, rlo, 6.702013582747528), rlo, -8.79639282735613), rlo, 5.629691409507923), rlo, -1.5833507089241035), rlo, 0.0), rlo, 0.07600083402835696))*rlo)*rlo);
  o.Lreg = -6.333402835696414*A[0] + 28.148457047539615*A[1] + -52.77835696413678*A[2] + 46.914095079232695*A[3] + -16.289616346955796*A[4];
  o.Preg = 0.07600083402835696*A[0] + -1.5833507089241035*A[2] + 5.629691409507923*A[3] + -8.79639282735613*A[4] + 6.702013582747528*A[5] + -2.0362020433694745*A[6];
  o.Mhat = -0.15200166805671392;
  o.MPhat = 0.0029314607410937687;
}
template <> __host__ __device__ __forceinline__ void Kern_quartic::adj<1>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = -12.666805671392828*A[0] + 84.44537114261885*A[1] + -211.11342785654713*A[2] + 234.57047539616346*A[3] + -97.73769808173478*A[4];
  const double a2 = -12.666805671392828*A[2] + 84.44537114261885*A[3] + -211.11342785654713*A[4] + 234.57047539616346*A[5] + -97.73769808173478*A[6];
  const double m1 = (((fma(fma(fma(fma(-16.289616346955796, rhi, 46.914095079232695), rhi, -52.77835696413678), rhi, 28.148457047539615), rhi, -6.333402835696414))*rhi)*rhi) - (((fma(fma(fma(fma(-16.289616346955796, rlo, 46.914095079232695), rlo, -52.77835696413678), rlo, 28.148457047539615), rlo, -6.333402835696414))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(-12.217212260216847, rhi, 33.510067913737636), rhi, -35.18557130942452), rhi, 16.88907422852377), rhi, -3.166701417848207))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(-12.217212260216847, rlo, 33.510067913737636), rlo, -35.18557130942452), rlo, 16.88907422852377), rlo, -3.166701417848207))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}
template <> __host__ __device__ __forceinline__ void Kern_quartic::sums<2>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1/5: P = ['375/1199', '-7500/1199', '56250/1199', '-187500/1199', '234375/1199']
  o.W0 = 0.3127606338615513*A[0] + -6.255212677231026*A[1] + 46.914095079232695*A[2] + -156.38031693077565*A[3] + 195.47539616346955*A[4];
  o.W1 = (((fma(fma(fma(fma(32.57923269391159, rhi, -31.27606338615513), rhi, 11.728523769808174), rhi, -2.085070892410342), rhi, 0.15638031693077564))*rhi)*rhi) - (((fma(fma(fma(fma(32.57923269391159, rlo, -31.27606338615513), rlo, 11.728523769808174), rlo, -2.085070892410342), rlo, 0.15638031693077564))*rlo)*rlo);
  o.P0 = -0.0004170141784820684*A[0] + 0.15638031693077564*A[2] + -2.085070892410342*A[3] + 11.728523769808174*A[4] + -31.27606338615513*A[5] + 32.57923269391159*A[6];
  o.P1 = (((fma(fma(fma(fma(fma(fma(4.072404086738949, rhi, -4.468009055165019), rhi, 1.9547539616346956), rhi, -0.4170141784820684), rhi, 0.03909507923269391), rhi, 0.0), rhi, -0.0002085070892410342))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(4.072404086738949, rlo, -4.468009055165019), rlo, 1.9547539616346956), rlo, -0.4170141784820684), rlo, 0.03909507923269391), rlo, 0.0), rlo, -0.0002085070892410342))*rlo)*rlo);
  o.Lreg = 0.15638031693077564*A[0] + -2.085070892410342*A[1] + 11.728523769808174*A[2] + -31.27606338615513*A[3] + 32.57923269391159*A[4];
  o.Preg = -0.0002085070892410342*A[0] + 0.03909507923269391*A[2] + -0.4170141784820684*A[3] + 1.9547539616346956*A[4] + -4.468009055165019*A[5] + 4.072404086738949*A[6];
  o.Mhat = 0.0004170141784820684;
  o.MPhat = -8.936018110330037e-07;
}
template <> __host__ __device__ __forceinline__ void Kern_quartic::adj<2>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 0.3127606338615513*A[0] + -6.255212677231026*A[1] + 46.914095079232695*A[2] + -156.38031693077565*A[3] + 195.47539616346955*A[4];
  const double a2 = 0.3127606338615513*A[2] + -6.255212677231026*A[3] + 46.914095079232695*A[4] + -156.38031693077565*A[5] + 195.47539616346955*A[6];
  const double m1 = (((fma(fma(fma(fma(32.57923269391159, rhi, -31.27606338615513), rhi, 11.728523769808174), rhi, -2.085070892410342), rhi, 0.15638031693077564))*rhi)*rhi) - (((fma(fma(fma(fma(32.57923269391159, rlo, -31.27606338615513), rlo, 11.728523769808174), rlo, -2.085070892410342), rlo, 0.15638031693077564))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(24.434424520433694, rhi, -22.34004527582509), rhi, 7.8190158465387825), rhi, -1.2510425354462051), rhi, 0.07819015846538782))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(24.434424520433694, rlo, -22.34004527582509), rlo, 7.8190158465387825), rlo, -1.2510425354462051), rlo, 0.07819015846538782))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- quintic: C2*pi = 15309/478, plane second moment 2771/51624
struct Kern_quintic {
  static constexpr int kId = 5;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 3;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.05367658453432512;
  static constexpr double kR[kBlocks] = {1.0, 0.6666666666666666, 0.3333333333333333};
  static constexpr int kNA[kBlocks] = {8, 8, 8};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {8, 8, 8};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_quintic::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['15309/478', '-76545/478', '76545/239', '-76545/239', '76545/478', '-15309/478']
  o.W0 = 32.02719665271967*A[0] + -160.13598326359832*A[1] + 320.27196652719664*A[2] + -320.27196652719664*A[3] + 160.13598326359832*A[4] + -32.02719665271967*A[5];
  o.W1 = (((fma(fma(fma(fma(fma(-4.575313807531381, rhi, 26.689330543933053), rhi, -64.05439330543933), rhi, 80.06799163179916), rhi, -53.37866108786611), rhi, 16.013598326359833))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-4.575313807531381, rlo, 26.689330543933053), rlo, -64.05439330543933), rlo, 80.06799163179916), rlo, -53.37866108786611), rlo, 16.013598326359833))*rlo)*rlo);
  o.P0 = -0.7625523012552301*A[0] + 16.013598326359833*A[2] + -53.37866108786611*A[3] + 80.06799163179916*A[4] + -64.05439330543933*A[5] + 26.689330543933053*A[6] + -4.575313807531381*A[7];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(-0.5083682008368201, rhi, 3.3361663179916317), rhi, -9.150627615062762), rhi, 13.344665271966527), rhi, -10.675732217573222), rhi, 4.003399581589958), rhi, 0.0), rhi, -0.38127615062761505))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(-0.5083682008368201, rlo, 3.3361663179916317), rlo, -9.150627615062762), rlo, 13.344665271966527), rlo, -10.675732217573222), rlo, 4.003399581589958), rlo, 0.0), rlo, -0.38127615062761505))*rlo)*rlo);
  o.Lreg = 16.013598326359833*A[0] + -53.37866108786611*A[1] + 80.06799163179916*A[2] + -64.05439330543933*A[3] + 26.689330543933053*A[4] + -4.575313807531381*A[5];
  o.Preg = -0.38127615062761505*A[0] + 4.003399581589958*A[2] + -10.675732217573222*A[3] + 13.344665271966527*A[4] + -9.150627615062762*A[5] + 3.3361663179916317*A[6] + -0.5083682008368201*A[7];
  o.Mhat = 0.7625523012552301;
  o.MPhat = -0.03177301255230126;
}
template <> __host__ __device__ __forceinline__ void Kern_quintic::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 32.02719665271967*A[0] + -160.13598326359832*A[1] + 320.27196652719664*A[2] + -320.27196652719664*A[3] + 160.13598326359832*A[4] + -32.02719665271967*A[5];
  const double a2 = 32.02719665271967*A[2] + -160.13598326359832*A[3] + 320.27196652719664*A[4] + -320.27196652719664*A[5] + 160.13598326359832*A[6] + -32.02719665271967*A[7];
  const double m1 = (((fma(fma(fma(fma(fma(-4.575313807531381, rhi, 26.689330543933053), rhi, -64.05439330543933), rhi, 80.06799163179916), rhi, -53.37866108786611), rhi, 16.013598326359833))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-4.575313807531381, rlo, 26.689330543933053), rlo, -64.05439330543933), rlo, 80.06799163179916), rlo, -53.37866108786611), rlo, 16.013598326359833))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(-3.5585774058577404, rhi, 20.01699790794979), rhi, -45.75313807531381), rhi, 53.37866108786611), rhi, -32.02719665271967), rhi, 8.006799163179917))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(-3.5585774058577404, rlo, 20.01699790794979), rlo, -45.75313807531381), rlo, 53.37866108786611), rlo, -32.02719665271967), rlo, 8.006799163179917))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}
template <> __host__ __device__ __forceinline__ void Kern_quintic::sums<1>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 2/3: P = ['-6048/239', '45360/239', '-136080/239', '204120/239', '-153090/239', '45927/239']
  o.W0 = -25.305439330543933*A[0] + 189.7907949790795*A[1] + -569.3723849372385*A[2] + 854.0585774058577*A[3] + -640.5439330543933*A[4] + 192.163179916318*A[5];
  o.W1 = (((fma(fma(fma(fma(fma(27.451882845188283, rhi, -106.75732217573221), rhi, 170.81171548117155), rhi, -142.34309623430963), rhi, 63.26359832635983), rhi, -12.652719665271967))*rhi)*rhi) - (((fma(fma(fma(fma(fma(27.451882845188283, rlo, -106.75732217573221), rlo, 170.81171548117155), rlo, -142.34309623430963), rlo, 63.26359832635983), rlo, -12.652719665271967))*rlo)*rlo);
  o.P0 = 0.26778242677824265*A[0] + -12.652719665271967*A[2] + 63.26359832635983*A[3] + -142.34309623430963*A[4] + 170.81171548117155*A[5] + -106.75732217573221*A[6] + 27.451882845188283*A[7];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(3.0502092050209204, rhi, -13.344665271966527), rhi, 24.401673640167363), rhi, -23.723849372384937), rhi, 12.652719665271967), rhi, -3.1631799163179917), rhi, 0.0), rhi, 0.13389121338912133))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(3.0502092050209204, rlo, -13.344665271966527), rlo, 24.401673640167363), rlo, -23.723849372384937), rlo, 12.652719665271967), rlo, -3.1631799163179917), rlo, 0.0), rlo, 0.13389121338912133))*rlo)*rlo);
  o.Lreg = -12.652719665271967*A[0] + 63.26359832635983*A[1] + -142.34309623430963*A[2] + 170.81171548117155*A[3] + -106.75732217573221*A[4] + 27.451882845188283*A[5];
  o.Preg = 0.13389121338912133*A[0] + -3.1631799163179917*A[2] + 12.652719665271967*A[3] + -23.723849372384937*A[4] + 24.401673640167363*A[5] + -13.344665271966527*A[6] + 3.0502092050209204*A[7];
  o.Mhat = -0.26778242677824265;
  o.MPhat = 0.004958933829226716;
}
template <> __host__ __device__ __forceinline__ void Kern_quintic::adj<1>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = -25.305439330543933*A[0] + 189.7907949790795*A[1] + -569.3723849372385*A[2] + 854.0585774058577*A[3] + -640.5439330543933*A[4] + 192.163179916318*A[5];
  const double a2 = -25.305439330543933*A[2] + 189.7907949790795*A[3] + -569.3723849372385*A[4] + 854.0585774058577*A[5] + -640.5439330543933*A[6] + 192.163179916318*A[7];
  const double m1 = (((fma(fma(fma(fma(fma(27.451882845188283, rhi, -106.75732217573221), rhi, 170.81171548117155), rhi, -142.34309623430963), rhi, 63.26359832635983), rhi, -12.652719665271967))*rhi)*rhi) - (((fma(fma(fma(fma(fma(27.451882845188283, rlo, -106.75732217573221), rlo, 170.81171548117155), rlo, -142.34309623430963), rlo, 63.26359832635983), rlo, -12.652719665271967))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(21.351464435146443, rhi, -80.06799163179916), rhi, 122.00836820083683), rhi, -94.89539748953975), rhi, 37.9581589958159), rhi, -6.326359832635983))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(21.351464435146443, rlo, -80.06799163179916), rlo, 122.00836820083683), rlo, -94.89539748953975), rlo, 37.9581589958159), rlo, -6.326359832635983))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}
template <> __host__ __device__ __forceinline__ void Kern_quintic::sums<2>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1/3: P = ['945/478', '-14175/478', '42525/239', '-127575/239', '382725/478', '-229635/478']
  o.W0 = 1.9769874476987448*A[0] + -29.65481171548117*A[1] + 177.92887029288704*A[2] + -533.7866108786611*A[3] + 800.6799163179917*A[4] + -480.407949790795*A[5];
  o.W1 = (((fma(fma(fma(fma(fma(-68.6297071129707, rhi, 133.44665271966528), rhi, -106.75732217573221), rhi, 44.48221757322176), rhi, -9.884937238493723), rhi, 0.9884937238493724))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-68.6297071129707, rlo, 133.44665271966528), rlo, -106.75732217573221), rlo, 44.48221757322176), rlo, -9.884937238493723), rlo, 0.9884937238493724))*rlo)*rlo);
  o.P0 = -0.005230125523012552*A[0] + 0.9884937238493724*A[2] + -9.884937238493723*A[3] + 44.48221757322176*A[4] + -106.75732217573221*A[5] + 133.44665271966528*A[6] + -68.6297071129707*A[7];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(-7.625523012552302, rhi, 16.68083158995816), rhi, -15.251046025104603), rhi, 7.4137029288702925), rhi, -1.9769874476987448), rhi, 0.2471234309623431), rhi, 0.0), rhi, -0.002615062761506276))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(-7.625523012552302, rlo, 16.68083158995816), rlo, -15.251046025104603), rlo, 7.4137029288702925), rlo, -1.9769874476987448), rlo, 0.2471234309623431), rlo, 0.0), rlo, -0.002615062761506276))*rlo)*rlo);
  o.Lreg = 0.9884937238493724*A[0] + -9.884937238493723*A[1] + 44.48221757322176*A[2] + -106.75732217573221*A[3] + 133.44665271966528*A[4] + -68.6297071129707*A[5];
  o.Preg = -0.002615062761506276*A[0] + 0.2471234309623431*A[2] + -1.9769874476987448*A[3] + 7.4137029288702925*A[4] + -15.251046025104603*A[5] + 16.68083158995816*A[6] + -7.625523012552302*A[7];
  o.Mhat = 0.005230125523012552;
  o.MPhat = -2.4213544088021077e-05;
}
template <> __host__ __device__ __forceinline__ void Kern_quintic::adj<2>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 1.9769874476987448*A[0] + -29.65481171548117*A[1] + 177.92887029288704*A[2] + -533.7866108786611*A[3] + 800.6799163179917*A[4] + -480.407949790795*A[5];
  const double a2 = 1.9769874476987448*A[2] + -29.65481171548117*A[3] + 177.92887029288704*A[4] + -533.7866108786611*A[5] + 800.6799163179917*A[6] + -480.407949790795*A[7];
  const double m1 = (((fma(fma(fma(fma(fma(-68.6297071129707, rhi, 133.44665271966528), rhi, -106.75732217573221), rhi, 44.48221757322176), rhi, -9.884937238493723), rhi, 0.9884937238493724))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-68.6297071129707, rlo, 133.44665271966528), rlo, -106.75732217573221), rlo, 44.48221757322176), rlo, -9.884937238493723), rlo, 0.9884937238493724))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(-53.37866108786611, rhi, 100.08498953974896), rhi, -76.25523012552301), rhi, 29.65481171548117), rhi, -5.930962343096234), rhi, 0.4942468619246862))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(-53.37866108786611, rlo, 100.08498953974896), rlo, -76.25523012552301), rlo, 29.65481171548117), rlo, -5.930962343096234), rlo, 0.4942468619246862))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- poly6: C2*pi = 4, plane second moment 1/10
struct Kern_poly6 {
  static constexpr int kId = 6;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.1;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {9};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {9};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_poly6::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['4', '0', '-12', '0', '12', '0', '-4']
  o.W0 = 4.0*A[0] + -12.0*A[2] + 12.0*A[4] + -4.0*A[6];
  o.W1 = (((fma(fma(fma(fma(fma(fma(-0.5, rhi, 0.0), rhi, 2.0), rhi, 0.0), rhi, -3.0), rhi, 0.0), rhi, 2.0))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(-0.5, rlo, 0.0), rlo, 2.0), rlo, 0.0), rlo, -3.0), rlo, 0.0), rlo, 2.0))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 2.0*A[2] + -3.0*A[4] + 2.0*A[6] + -0.5*A[8];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(fma(-0.05, rhi, 0.0), rhi, 0.25), rhi, 0.0), rhi, -0.5), rhi, 0.0), rhi, 0.5), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(-0.05, rlo, 0.0), rlo, 0.25), rlo, 0.0), rlo, -0.5), rlo, 0.0), rlo, 0.5), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 2.0*A[0] + -3.0*A[2] + 2.0*A[4] + -0.5*A[6];
  o.Preg = -0.25*A[0] + 0.5*A[2] + -0.5*A[4] + 0.25*A[6] + -0.05*A[8];
  o.Mhat = 0.5;
  o.MPhat = -0.05;
}
template <> __host__ __device__ __forceinline__ void Kern_poly6::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 4.0*A[0] + -12.0*A[2] + 12.0*A[4] + -4.0*A[6];
  const double a2 = 4.0*A[2] + -12.0*A[4] + 12.0*A[6] + -4.0*A[8];
  const double m1 = (((fma(fma(fma(fma(fma(fma(-0.5, rhi, 0.0), rhi, 2.0), rhi, 0.0), rhi, -3.0), rhi, 0.0), rhi, 2.0))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(-0.5, rlo, 0.0), rlo, 2.0), rlo, 0.0), rlo, -3.0), rlo, 0.0), rlo, 2.0))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(fma(-0.4, rhi, 0.0), rhi, 1.5), rhi, 0.0), rhi, -2.0), rhi, 0.0), rhi, 1.0))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(fma(-0.4, rlo, 0.0), rlo, 1.5), rlo, 0.0), rlo, -2.0), rlo, 0.0), rlo, 1.0))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- cone: C2*pi = 3, plane second moment 3/20
struct Kern_cone {
  static constexpr int kId = 7;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.15;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {4};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {4};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_cone::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['3', '-3']
  o.W0 = 3.0*A[0] + -3.0*A[1];
  o.W1 = (((fma(-1.0, rhi, 1.5))*rhi)*rhi) - (((fma(-1.0, rlo, 1.5))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 1.5*A[2] + -1.0*A[3];
  o.P1 = (((fma(fma(fma(-0.2, rhi, 0.375), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(-0.2, rlo, 0.375), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 1.5*A[0] + -1.0*A[1];
  o.Preg = -0.25*A[0] + 0.375*A[2] + -0.2*A[3];
  o.Mhat = 0.5;
  o.MPhat = -0.075;
}
template <> __host__ __device__ __forceinline__ void Kern_cone::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 3.0*A[0] + -3.0*A[1];
  const double a2 = 3.0*A[2] + -3.0*A[3];
  const double m1 = (((fma(-1.0, rhi, 1.5))*rhi)*rhi) - (((fma(-1.0, rlo, 1.5))*rlo)*rlo);
  const double m3 = (((((fma(-0.6, rhi, 0.75))*rhi)*rhi)*rhi)*rhi) - (((((fma(-0.6, rlo, 0.75))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- lw2: C2*pi = 10, plane second moment 1/14
struct Kern_lw2 {
  static constexpr int kId = 8;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.07142857142857142;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {6};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {6};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_lw2::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['10', '-30', '30', '-10']
  o.W0 = 10.0*A[0] + -30.0*A[1] + 30.0*A[2] + -10.0*A[3];
  o.W1 = (((fma(fma(fma(-2.0, rhi, 7.5), rhi, -10.0), rhi, 5.0))*rhi)*rhi) - (((fma(fma(fma(-2.0, rlo, 7.5), rlo, -10.0), rlo, 5.0))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 5.0*A[2] + -10.0*A[3] + 7.5*A[4] + -2.0*A[5];
  o.P1 = (((fma(fma(fma(fma(fma(-0.2857142857142857, rhi, 1.25), rhi, -2.0), rhi, 1.25), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(-0.2857142857142857, rlo, 1.25), rlo, -2.0), rlo, 1.25), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 5.0*A[0] + -10.0*A[1] + 7.5*A[2] + -2.0*A[3];
  o.Preg = -0.25*A[0] + 1.25*A[2] + -2.0*A[3] + 1.25*A[4] + -0.2857142857142857*A[5];
  o.Mhat = 0.5;
  o.MPhat = -0.03571428571428571;
}
template <> __host__ __device__ __forceinline__ void Kern_lw2::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 10.0*A[0] + -30.0*A[1] + 30.0*A[2] + -10.0*A[3];
  const double a2 = 10.0*A[2] + -30.0*A[3] + 30.0*A[4] + -10.0*A[5];
  const double m1 = (((fma(fma(fma(-2.0, rhi, 7.5), rhi, -10.0), rhi, 5.0))*rhi)*rhi) - (((fma(fma(fma(-2.0, rlo, 7.5), rlo, -10.0), rlo, 5.0))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(-1.4285714285714286, rhi, 5.0), rhi, -6.0), rhi, 2.5))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(-1.4285714285714286, rlo, 5.0), rlo, -6.0), rlo, 2.5))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- lw4: C2*pi = 28/3, plane second moment 1/18
struct Kern_lw4 {
  static constexpr int kId = 9;
  static constexpr bool kQuad = false;
  static constexpr int kBlocks = 1;
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.05555555555555555;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {9};   // A_0..A_{kNA-1} for the forward sums
  static constexpr int kNAadj[kBlocks] = {9};   // for the adjoint sums
  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);
  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);
};
template <> __host__ __device__ __forceinline__ void Kern_lw4::sums<0>(const double* A, double rlo, double rhi, BlockSums& o) {
  // block R = 1: P = ['28/3', '0', '-140', '1120/3', '-420', '224', '-140/3']
  o.W0 = 9.333333333333334*A[0] + -140.0*A[2] + 373.3333333333333*A[3] + -420.0*A[4] + 224.0*A[5] + -46.666666666666664*A[6];
  o.W1 = (((fma(fma(fma(fma(fma(fma(-5.833333333333333, rhi, 32.0), rhi, -70.0), rhi, 74.66666666666667), rhi, -35.0), rhi, 0.0), rhi, 4.666666666666667))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(-5.833333333333333, rlo, 32.0), rlo, -70.0), rlo, 74.66666666666667), rlo, -35.0), rlo, 0.0), rlo, 4.666666666666667))*rlo)*rlo);
  o.P0 = -0.5*A[0] + 4.666666666666667*A[2] + -35.0*A[4] + 74.66666666666667*A[5] + -70.0*A[6] + 32.0*A[7] + -5.833333333333333*A[8];
  o.P1 = (((fma(fma(fma(fma(fma(fma(fma(fma(-0.5833333333333334, rhi, 3.5555555555555554), rhi, -8.75), rhi, 10.666666666666666), rhi, -5.833333333333333), rhi, 0.0), rhi, 1.1666666666666667), rhi, 0.0), rhi, -0.25))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(fma(fma(-0.5833333333333334, rlo, 3.5555555555555554), rlo, -8.75), rlo, 10.666666666666666), rlo, -5.833333333333333), rlo, 0.0), rlo, 1.1666666666666667), rlo, 0.0), rlo, -0.25))*rlo)*rlo);
  o.Lreg = 4.666666666666667*A[0] + -35.0*A[2] + 74.66666666666667*A[3] + -70.0*A[4] + 32.0*A[5] + -5.833333333333333*A[6];
  o.Preg = -0.25*A[0] + 1.1666666666666667*A[2] + -5.833333333333333*A[4] + 10.666666666666666*A[5] + -8.75*A[6] + 3.5555555555555554*A[7] + -0.5833333333333334*A[8];
  o.Mhat = 0.5;
  o.MPhat = -0.027777777777777776;
}
template <> __host__ __device__ __forceinline__ void Kern_lw4::adj<0>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {
  const double a0 = 9.333333333333334*A[0] + -140.0*A[2] + 373.3333333333333*A[3] + -420.0*A[4] + 224.0*A[5] + -46.666666666666664*A[6];
  const double a2 = 9.333333333333334*A[2] + -140.0*A[4] + 373.3333333333333*A[5] + -420.0*A[6] + 224.0*A[7] + -46.666666666666664*A[8];
  const double m1 = (((fma(fma(fma(fma(fma(fma(-5.833333333333333, rhi, 32.0), rhi, -70.0), rhi, 74.66666666666667), rhi, -35.0), rhi, 0.0), rhi, 4.666666666666667))*rhi)*rhi) - (((fma(fma(fma(fma(fma(fma(-5.833333333333333, rlo, 32.0), rlo, -70.0), rlo, 74.66666666666667), rlo, -35.0), rlo, 0.0), rlo, 4.666666666666667))*rlo)*rlo);
  const double m3 = (((((fma(fma(fma(fma(fma(fma(-4.666666666666667, rhi, 24.88888888888889), rhi, -52.5), rhi, 53.333333333333336), rhi, -23.333333333333332), rhi, 0.0), rhi, 2.3333333333333335))*rhi)*rhi)*rhi)*rhi) - (((((fma(fma(fma(fma(fma(fma(-4.666666666666667, rlo, 24.88888888888889), rlo, -52.5), rlo, 53.333333333333336), rlo, -23.333333333333332), rlo, 0.0), rlo, 2.3333333333333335))*rlo)*rlo)*rlo)*rlo);
  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;
}

// ---- reference term plans (plain FP64 interpreter): per kernel offsets into flat tables
constexpr int kPlanEdgeTerms = 165;
constexpr int kPlanValueTerms = 75;
constexpr int kPlanCoeffs = 1353;
constexpr int kPlanNumRadii = 15;
struct PlanOffsets { int e0, e1, v0, v1; };
static const PlanOffsets kPlanOffsets[kNumKernels] = {{0, 22, 0, 10}, {22, 33, 10, 15}, {33, 44, 15, 20}, {44, 55, 20, 25}, {55, 88, 25, 40}, {88, 121, 40, 55}, {121, 132, 55, 60}, {132, 143, 60, 65}, {143, 154, 65, 70}, {154, 165, 70, 75}};
static const int kPlanE[kPlanEdgeTerms][7] = {   // ch, i, a, b, radius index, c0, c1
  {1, 0, 0, 0, 0, 8, 13},
  {1, 0, 0, 0, 1, 13, 18},
  {2, 1, 0, 0, 0, 18, 23},
  {2, 1, 0, 0, 1, 23, 28},
  {3, 0, 0, 0, 0, 28, 32},
  {3, 0, 0, 0, 1, 32, 36},
  {4, 1, 0, 0, 0, 36, 40},
  {4, 1, 0, 0, 1, 40, 44},
  {5, 0, 1, 0, 0, 44, 48},
  {5, 0, 1, 0, 1, 48, 52},
  {6, 1, 1, 0, 0, 60, 64},
  {6, 1, 1, 0, 1, 64, 68},
  {7, 0, 0, 1, 0, 68, 72},
  {7, 0, 0, 1, 1, 72, 76},
  {8, 1, 0, 1, 0, 76, 80},
  {8, 1, 0, 1, 1, 80, 84},
  {9, 0, 1, 0, 0, 92, 97},
  {9, 0, 1, 0, 1, 97, 102},
  {10, 0, 0, 1, 0, 112, 117},
  {10, 0, 0, 1, 1, 117, 122},
  {11, 1, 0, 1, 0, 122, 127},
  {11, 1, 0, 1, 1, 127, 132},
  {1, 0, 0, 0, 2, 147, 153},
  {2, 1, 0, 0, 2, 153, 159},
  {3, 0, 0, 0, 2, 159, 164},
  {4, 1, 0, 0, 2, 164, 169},
  {5, 0, 1, 0, 2, 169, 174},
  {6, 1, 1, 0, 2, 179, 184},
  {7, 0, 0, 1, 2, 184, 189},
  {8, 1, 0, 1, 2, 189, 194},
  {9, 0, 1, 0, 2, 199, 205},
  {10, 0, 0, 1, 2, 211, 217},
  {11, 1, 0, 1, 2, 217, 223},
  {1, 0, 0, 0, 3, 236, 244},
  {2, 1, 0, 0, 3, 244, 252},
  {3, 0, 0, 0, 3, 252, 259},
  {4, 1, 0, 0, 3, 259, 266},
  {5, 0, 1, 0, 3, 266, 273},
  {6, 1, 1, 0, 3, 280, 287},
  {7, 0, 0, 1, 3, 287, 294},
  {8, 1, 0, 1, 3, 294, 301},
  {9, 0, 1, 0, 3, 308, 316},
  {10, 0, 0, 1, 3, 324, 332},
  {11, 1, 0, 1, 3, 332, 340},
  {1, 0, 0, 0, 4, 357, 367},
  {2, 1, 0, 0, 4, 367, 377},
  {3, 0, 0, 0, 4, 377, 386},
  {4, 1, 0, 0, 4, 386, 395},
  {5, 0, 1, 0, 4, 395, 404},
  {6, 1, 1, 0, 4, 413, 422},
  {7, 0, 0, 1, 4, 422, 431},
  {8, 1, 0, 1, 4, 431, 440},
  {9, 0, 1, 0, 4, 449, 459},
  {10, 0, 0, 1, 4, 469, 479},
  {11, 1, 0, 1, 4, 479, 489},
  {1, 0, 0, 0, 5, 514, 520},
  {1, 0, 0, 0, 6, 520, 526},
  {1, 0, 0, 0, 7, 526, 532},
  {2, 1, 0, 0, 5, 532, 538},
  {2, 1, 0, 0, 6, 538, 544},
  {2, 1, 0, 0, 7, 544, 550},
  {3, 0, 0, 0, 5, 550, 555},
  {3, 0, 0, 0, 6, 555, 560},
  {3, 0, 0, 0, 7, 560, 565},
  {4, 1, 0, 0, 5, 565, 570},
  {4, 1, 0, 0, 6, 570, 575},
  {4, 1, 0, 0, 7, 575, 580},
  {5, 0, 1, 0, 5, 580, 585},
  {5, 0, 1, 0, 6, 585, 590},
  {5, 0, 1, 0, 7, 590, 595},
  {6, 1, 1, 0, 5, 610, 615},
  {6, 1, 1, 0, 6, 615, 620},
  {6, 1, 1, 0, 7, 620, 625},
  {7, 0, 0, 1, 5, 625, 630},
  {7, 0, 0, 1, 6, 630, 635},
  {7, 0, 0, 1, 7, 635, 640},
  {8, 1, 0, 1, 5, 640, 645},
  {8, 1, 0, 1, 6, 645, 650},
  {8, 1, 0, 1, 7, 650, 655},
  {9, 0, 1, 0, 5, 670, 676},
  {9, 0, 1, 0, 6, 676, 682},
  {9, 0, 1, 0, 7, 682, 688},
  {10, 0, 0, 1, 5, 706, 712},
  {10, 0, 0, 1, 6, 712, 718},
  {10, 0, 0, 1, 7, 718, 724},
  {11, 1, 0, 1, 5, 724, 730},
  {11, 1, 0, 1, 6, 730, 736},
  {11, 1, 0, 1, 7, 736, 742},
  {1, 0, 0, 0, 8, 778, 785},
  {1, 0, 0, 0, 9, 785, 792},
  {1, 0, 0, 0, 10, 792, 799},
  {2, 1, 0, 0, 8, 799, 806},
  {2, 1, 0, 0, 9, 806, 813},
  {2, 1, 0, 0, 10, 813, 820},
  {3, 0, 0, 0, 8, 820, 826},
  {3, 0, 0, 0, 9, 826, 832},
  {3, 0, 0, 0, 10, 832, 838},
  {4, 1, 0, 0, 8, 838, 844},
  {4, 1, 0, 0, 9, 844, 850},
  {4, 1, 0, 0, 10, 850, 856},
  {5, 0, 1, 0, 8, 856, 862},
  {5, 0, 1, 0, 9, 862, 868},
  {5, 0, 1, 0, 10, 868, 874},
  {6, 1, 1, 0, 8, 892, 898},
  {6, 1, 1, 0, 9, 898, 904},
  {6, 1, 1, 0, 10, 904, 910},
  {7, 0, 0, 1, 8, 910, 916},
  {7, 0, 0, 1, 9, 916, 922},
  {7, 0, 0, 1, 10, 922, 928},
  {8, 1, 0, 1, 8, 928, 934},
  {8, 1, 0, 1, 9, 934, 940},
  {8, 1, 0, 1, 10, 940, 946},
  {9, 0, 1, 0, 8, 964, 971},
  {9, 0, 1, 0, 9, 971, 978},
  {9, 0, 1, 0, 10, 978, 985},
  {10, 0, 0, 1, 8, 1006, 1013},
  {10, 0, 0, 1, 9, 1013, 1020},
  {10, 0, 0, 1, 10, 1020, 1027},
  {11, 1, 0, 1, 8, 1027, 1034},
  {11, 1, 0, 1, 9, 1034, 1041},
  {11, 1, 0, 1, 10, 1041, 1048},
  {1, 0, 0, 0, 11, 1073, 1078},
  {2, 1, 0, 0, 11, 1078, 1083},
  {3, 0, 0, 0, 11, 1083, 1087},
  {4, 1, 0, 0, 11, 1087, 1091},
  {5, 0, 1, 0, 11, 1091, 1095},
  {6, 1, 1, 0, 11, 1099, 1103},
  {7, 0, 0, 1, 11, 1103, 1107},
  {8, 1, 0, 1, 11, 1107, 1111},
  {9, 0, 1, 0, 11, 1115, 1120},
  {10, 0, 0, 1, 11, 1125, 1130},
  {11, 1, 0, 1, 11, 1130, 1135},
  {1, 0, 0, 0, 12, 1142, 1145},
  {2, 1, 0, 0, 12, 1145, 1148},
  {3, 0, 0, 0, 12, 1148, 1150},
  {4, 1, 0, 0, 12, 1150, 1152},
  {5, 0, 1, 0, 12, 1152, 1154},
  {6, 1, 1, 0, 12, 1156, 1158},
  {7, 0, 0, 1, 12, 1158, 1160},
  {8, 1, 0, 1, 12, 1160, 1162},
  {9, 0, 1, 0, 12, 1164, 1167},
  {10, 0, 0, 1, 12, 1170, 1173},
  {11, 1, 0, 1, 12, 1173, 1176},
  {1, 0, 0, 0, 13, 1183, 1188},
  {2, 1, 0, 0, 13, 1188, 1193},
  {3, 0, 0, 0, 13, 1193, 1197},
  {4, 1, 0, 0, 13, 1197, 1201},
  {5, 0, 1, 0, 13, 1201, 1205},
  {6, 1, 1, 0, 13, 1209, 1213},
  {7, 0, 0, 1, 13, 1213, 1217},
  {8, 1, 0, 1, 13, 1217, 1221},
  {9, 0, 1, 0, 13, 1225, 1230},
  {10, 0, 0, 1, 13, 1235, 1240},
  {11, 1, 0, 1, 13, 1240, 1245},
  {1, 0, 0, 0, 14, 1256, 1263},
  {2, 1, 0, 0, 14, 1263, 1270},
  {3, 0, 0, 0, 14, 1270, 1276},
  {4, 1, 0, 0, 14, 1276, 1282},
  {5, 0, 1, 0, 14, 1282, 1288},
  {6, 1, 1, 0, 14, 1294, 1300},
  {7, 0, 0, 1, 14, 1300, 1306},
  {8, 1, 0, 1, 14, 1306, 1312},
  {9, 0, 1, 0, 14, 1318, 1325},
  {10, 0, 0, 1, 14, 1332, 1339},
  {11, 1, 0, 1, 14, 1339, 1346},
};
static const int kPlanVi[kPlanValueTerms][4] = {   // ch, radius index, c0, c1
  {0, 0, 0, 4},
  {0, 1, 4, 8},
  {5, 0, 52, 56},
  {5, 1, 56, 60},
  {8, 0, 84, 88},
  {8, 1, 88, 92},
  {9, 0, 102, 107},
  {9, 1, 107, 112},
  {11, 0, 132, 137},
  {11, 1, 137, 142},
  {0, 2, 142, 147},
  {5, 2, 174, 179},
  {8, 2, 194, 199},
  {9, 2, 205, 211},
  {11, 2, 223, 229},
  {0, 3, 229, 236},
  {5, 3, 273, 280},
  {8, 3, 301, 308},
  {9, 3, 316, 324},
  {11, 3, 340, 348},
  {0, 4, 348, 357},
  {5, 4, 404, 413},
  {8, 4, 440, 449},
  {9, 4, 459, 469},
  {11, 4, 489, 499},
  {0, 5, 499, 504},
  {0, 6, 504, 509},
  {0, 7, 509, 514},
  {5, 5, 595, 600},
  {5, 6, 600, 605},
  {5, 7, 605, 610},
  {8, 5, 655, 660},
  {8, 6, 660, 665},
  {8, 7, 665, 670},
  {9, 5, 688, 694},
  {9, 6, 694, 700},
  {9, 7, 700, 706},
  {11, 5, 742, 748},
  {11, 6, 748, 754},
  {11, 7, 754, 760},
  {0, 8, 760, 766},
  {0, 9, 766, 772},
  {0, 10, 772, 778},
  {5, 8, 874, 880},
  {5, 9, 880, 886},
  {5, 10, 886, 892},
  {8, 8, 946, 952},
  {8, 9, 952, 958},
  {8, 10, 958, 964},
  {9, 8, 985, 992},
  {9, 9, 992, 999},
  {9, 10, 999, 1006},
  {11, 8, 1048, 1055},
  {11, 9, 1055, 1062},
  {11, 10, 1062, 1069},
  {0, 11, 1069, 1073},
  {5, 11, 1095, 1099},
  {8, 11, 1111, 1115},
  {9, 11, 1120, 1125},
  {11, 11, 1135, 1140},
  {0, 12, 1140, 1142},
  {5, 12, 1154, 1156},
  {8, 12, 1162, 1164},
  {9, 12, 1167, 1170},
  {11, 12, 1176, 1179},
  {0, 13, 1179, 1183},
  {5, 13, 1205, 1209},
  {8, 13, 1221, 1225},
  {9, 13, 1230, 1235},
  {11, 13, 1245, 1250},
  {0, 14, 1250, 1256},
  {5, 14, 1288, 1294},
  {8, 14, 1312, 1318},
  {9, 14, 1325, 1332},
  {11, 14, 1346, 1353},
};
static const double kPlanVmR[kPlanValueTerms] = {0.5714285714285714, -0.07142857142857142, 0.5714285714285714, -0.07142857142857142, 0.5714285714285714, -0.07142857142857142, 0.04081632653061224, -0.0012755102040816326, 0.04081632653061224, -0.0012755102040816326, 0.5, 0.5, 0.5, 0.034722222222222224, 0.034722222222222224, 0.5, 0.5, 0.5, 0.026515151515151516, 0.026515151515151516, 0.5, 0.5, 0.5, 0.02142857142857143, 0.02142857142857143, 0.6515846538782318, -0.15200166805671392, 0.0004170141784820684, 0.6515846538782318, -0.15200166805671392, 0.0004170141784820684, 0.6515846538782318, -0.15200166805671392, 0.0004170141784820684, 0.03490632074347671, -0.0029314607410937687, 8.936018110330037e-07, 0.03490632074347671, -0.0029314607410937687, 8.936018110330037e-07, 0.7625523012552301, -0.26778242677824265, 0.005230125523012552, 0.7625523012552301, -0.26778242677824265, 0.005230125523012552, 0.7625523012552301, -0.26778242677824265, 0.005230125523012552, 0.03177301255230126, -0.004958933829226716, 2.4213544088021077e-05, 0.03177301255230126, -0.004958933829226716, 2.4213544088021077e-05, 0.5, 0.5, 0.5, 0.05, 0.05, 0.5, 0.5, 0.5, 0.075, 0.075, 0.5, 0.5, 0.5, 0.03571428571428571, 0.03571428571428571, 0.5, 0.5, 0.5, 0.027777777777777776, 0.027777777777777776};
static const int kPlanCn[kPlanCoeffs] = {0, 1, 2, 3, 0, 1, 2, 3, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 7, 8, 9, 10, 11, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 2, 4, 6, 8, 9, 10, 11, 12, 13, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 1, 2, 3, 4, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 1, 2, 3, 4, 5, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 3, 4, 5, 6, 7, 0, 2, 4, 6, 0, 2, 4, 6, 8, 0, 2, 4, 6, 8, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 0, 2, 4, 6, 8, 0, 2, 4, 6, 8, 0, 2, 4, 6, 8, 0, 2, 4, 6, 8, 0, 2, 4, 6, 8, 0, 1, 0, 2, 3, 0, 2, 3, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 2, 3, 0, 2, 3, 0, 2, 3, 0, 2, 3, 0, 2, 3, 0, 1, 2, 3, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 1, 2, 3, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 0, 2, 3, 4, 5, 6, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 3, 4, 5, 6, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8, 0, 2, 4, 5, 6, 7, 8};
static const double kPlanCc[kPlanCoeffs] = {5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -0.5714285714285714, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, 0.07142857142857142, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -0.5714285714285714, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, 0.07142857142857142, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, -11.428571428571429, 34.285714285714285, -34.285714285714285, 11.428571428571429, 5.714285714285714, -34.285714285714285, 68.57142857142857, -45.714285714285715, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -0.5714285714285714, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, 0.07142857142857142, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, 0.2857142857142857, -1.4285714285714286, 2.2857142857142856, -1.4285714285714286, 0.32653061224489793, -0.03571428571428571, 0.7142857142857143, -2.2857142857142856, 2.857142857142857, -1.3061224489795917, -0.5714285714285714, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, 0.07142857142857142, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, -0.5714285714285714, 5.714285714285714, -11.428571428571429, 8.571428571428571, -2.2857142857142856, 0.07142857142857142, -2.857142857142857, 11.428571428571429, -17.142857142857142, 9.142857142857142, 0.2857142857142857, -1.4285714285714286, 2.2857142857142856, -1.4285714285714286, 0.32653061224489793, -0.03571428571428571, 0.7142857142857143, -2.2857142857142856, 2.857142857142857, -1.3061224489795917, 3.5, -17.5, 28.0, -17.5, 4.0, -0.5, 3.5, -17.5, 28.0, -17.5, 4.0, -0.5, 3.5, -17.5, 28.0, -17.5, 4.0, -7.0, 70.0, -140.0, 105.0, -28.0, -7.0, 70.0, -140.0, 105.0, -28.0, -7.0, 70.0, -140.0, 105.0, -28.0, 3.5, -17.5, 28.0, -17.5, 4.0, -7.0, 70.0, -140.0, 105.0, -28.0, -7.0, 70.0, -140.0, 105.0, -28.0, -7.0, 70.0, -140.0, 105.0, -28.0, 3.5, -17.5, 28.0, -17.5, 4.0, -0.5, 3.5, -17.5, 28.0, -17.5, 4.0, 0.25, -0.875, 2.9166666666666665, -4.0, 2.1875, -0.4444444444444444, -0.5, 3.5, -17.5, 28.0, -17.5, 4.0, -0.5, 3.5, -17.5, 28.0, -17.5, 4.0, 0.25, -0.875, 2.9166666666666665, -4.0, 2.1875, -0.4444444444444444, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -0.5, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -0.5, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, -9.0, 84.0, -630.0, 1344.0, -1260.0, 576.0, -105.0, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -0.5, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, 0.25, -1.125, 3.5, -13.125, 21.333333333333332, -15.75, 5.818181818181818, -0.875, -0.5, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, -0.5, 4.5, -21.0, 105.0, -192.0, 157.5, -64.0, 10.5, 0.25, -1.125, 3.5, -13.125, 21.333333333333332, -15.75, 5.818181818181818, -0.875, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -0.5, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -0.5, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, -11.142857142857142, 122.57142857142857, -735.4285714285714, 5148.0, -11766.857142857143, 12870.0, -7844.571428571428, 2574.0, -356.57142857142856, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -0.5, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, 0.25, -1.3928571428571428, 5.107142857142857, -15.321428571428571, 64.35, -118.85714285714286, 107.25, -54.857142857142854, 15.321428571428571, -1.8285714285714285, -0.5, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, -0.5, 5.571428571428571, -30.642857142857142, 122.57142857142857, -643.5, 1307.4285714285713, -1287.0, 713.1428571428571, -214.5, 27.428571428571427, 0.25, -1.3928571428571428, 5.107142857142857, -15.321428571428571, 64.35, -118.85714285714286, 107.25, -54.857142857142854, 15.321428571428571, -1.8285714285714285, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -0.6515846538782318, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, 0.15200166805671392, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, -0.0004170141784820684, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -0.6515846538782318, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, 0.15200166805671392, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, -0.0004170141784820684, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, -19.547539616346956, 78.19015846538782, -117.28523769808173, 78.19015846538782, -19.547539616346956, 12.666805671392828, -84.44537114261885, 211.11342785654713, -234.57047539616346, 97.73769808173478, -0.3127606338615513, 6.255212677231026, -46.914095079232695, 156.38031693077565, -195.47539616346955, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -0.6515846538782318, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, 0.15200166805671392, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, -0.0004170141784820684, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, 0.3257923269391159, -2.4434424520433695, 5.212677231025855, -4.886884904086739, 2.2340045275825093, -0.40724040867389494, -0.07600083402835696, 1.5833507089241035, -5.629691409507923, 8.79639282735613, -6.702013582747528, 2.0362020433694745, 0.0002085070892410342, -0.03909507923269391, 0.4170141784820684, -1.9547539616346956, 4.468009055165019, -4.072404086738949, -0.6515846538782318, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, 0.15200166805671392, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, -0.0004170141784820684, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, -0.6515846538782318, 9.773769808173478, -26.063386155129276, 29.321309424520432, -15.638031693077565, 3.2579232693911595, 0.15200166805671392, -6.333402835696414, 28.148457047539615, -52.77835696413678, 46.914095079232695, -16.289616346955796, -0.0004170141784820684, 0.15638031693077564, -2.085070892410342, 11.728523769808174, -31.27606338615513, 32.57923269391159, 0.3257923269391159, -2.4434424520433695, 5.212677231025855, -4.886884904086739, 2.2340045275825093, -0.40724040867389494, -0.07600083402835696, 1.5833507089241035, -5.629691409507923, 8.79639282735613, -6.702013582747528, 2.0362020433694745, 0.0002085070892410342, -0.03909507923269391, 0.4170141784820684, -1.9547539616346956, 4.468009055165019, -4.072404086738949, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -0.7625523012552301, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, 0.26778242677824265, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, -0.005230125523012552, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -0.7625523012552301, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, 0.26778242677824265, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, -0.005230125523012552, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, -32.02719665271967, 160.13598326359832, -320.27196652719664, 320.27196652719664, -160.13598326359832, 32.02719665271967, 25.305439330543933, -189.7907949790795, 569.3723849372385, -854.0585774058577, 640.5439330543933, -192.163179916318, -1.9769874476987448, 29.65481171548117, -177.92887029288704, 533.7866108786611, -800.6799163179917, 480.407949790795, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -0.7625523012552301, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, 0.26778242677824265, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, -0.005230125523012552, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, 0.38127615062761505, -4.003399581589958, 10.675732217573222, -13.344665271966527, 9.150627615062762, -3.3361663179916317, 0.5083682008368201, -0.13389121338912133, 3.1631799163179917, -12.652719665271967, 23.723849372384937, -24.401673640167363, 13.344665271966527, -3.0502092050209204, 0.002615062761506276, -0.2471234309623431, 1.9769874476987448, -7.4137029288702925, 15.251046025104603, -16.68083158995816, 7.625523012552302, -0.7625523012552301, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, 0.26778242677824265, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, -0.005230125523012552, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, -0.7625523012552301, 16.013598326359833, -53.37866108786611, 80.06799163179916, -64.05439330543933, 26.689330543933053, -4.575313807531381, 0.26778242677824265, -12.652719665271967, 63.26359832635983, -142.34309623430963, 170.81171548117155, -106.75732217573221, 27.451882845188283, -0.005230125523012552, 0.9884937238493724, -9.884937238493723, 44.48221757322176, -106.75732217573221, 133.44665271966528, -68.6297071129707, 0.38127615062761505, -4.003399581589958, 10.675732217573222, -13.344665271966527, 9.150627615062762, -3.3361663179916317, 0.5083682008368201, -0.13389121338912133, 3.1631799163179917, -12.652719665271967, 23.723849372384937, -24.401673640167363, 13.344665271966527, -3.0502092050209204, 0.002615062761506276, -0.2471234309623431, 1.9769874476987448, -7.4137029288702925, 15.251046025104603, -16.68083158995816, 7.625523012552302, 2.0, -3.0, 2.0, -0.5, -0.5, 2.0, -3.0, 2.0, -0.5, -0.5, 2.0, -3.0, 2.0, -0.5, -4.0, 12.0, -12.0, 4.0, -4.0, 12.0, -12.0, 4.0, -4.0, 12.0, -12.0, 4.0, 2.0, -3.0, 2.0, -0.5, -4.0, 12.0, -12.0, 4.0, -4.0, 12.0, -12.0, 4.0, -4.0, 12.0, -12.0, 4.0, 2.0, -3.0, 2.0, -0.5, -0.5, 2.0, -3.0, 2.0, -0.5, 0.25, -0.5, 0.5, -0.25, 0.05, -0.5, 2.0, -3.0, 2.0, -0.5, -0.5, 2.0, -3.0, 2.0, -0.5, 0.25, -0.5, 0.5, -0.25, 0.05, 1.5, -1.0, -0.5, 1.5, -1.0, -0.5, 1.5, -1.0, -3.0, 3.0, -3.0, 3.0, -3.0, 3.0, 1.5, -1.0, -3.0, 3.0, -3.0, 3.0, -3.0, 3.0, 1.5, -1.0, -0.5, 1.5, -1.0, 0.25, -0.375, 0.2, -0.5, 1.5, -1.0, -0.5, 1.5, -1.0, 0.25, -0.375, 0.2, 5.0, -10.0, 7.5, -2.0, -0.5, 5.0, -10.0, 7.5, -2.0, -0.5, 5.0, -10.0, 7.5, -2.0, -10.0, 30.0, -30.0, 10.0, -10.0, 30.0, -30.0, 10.0, -10.0, 30.0, -30.0, 10.0, 5.0, -10.0, 7.5, -2.0, -10.0, 30.0, -30.0, 10.0, -10.0, 30.0, -30.0, 10.0, -10.0, 30.0, -30.0, 10.0, 5.0, -10.0, 7.5, -2.0, -0.5, 5.0, -10.0, 7.5, -2.0, 0.25, -1.25, 2.0, -1.25, 0.2857142857142857, -0.5, 5.0, -10.0, 7.5, -2.0, -0.5, 5.0, -10.0, 7.5, -2.0, 0.25, -1.25, 2.0, -1.25, 0.2857142857142857, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -0.5, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -0.5, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, -9.333333333333334, 140.0, -373.3333333333333, 420.0, -224.0, 46.666666666666664, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -0.5, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, 0.25, -1.1666666666666667, 5.833333333333333, -10.666666666666666, 8.75, -3.5555555555555554, 0.5833333333333334, -0.5, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, -0.5, 4.666666666666667, -35.0, 74.66666666666667, -70.0, 32.0, -5.833333333333333, 0.25, -1.1666666666666667, 5.833333333333333, -10.666666666666666, 8.75, -3.5555555555555554, 0.5833333333333334};
static const double kPlanRadii[kPlanNumRadii] = {1.0, 0.5, 1.0, 1.0, 1.0, 1.0, 0.6, 0.2, 1.0, 0.6666666666666666, 0.3333333333333333, 1.0, 1.0, 1.0, 1.0};

// x^N by squaring
template <int N>
__host__ __device__ __forceinline__ double qpow(double x) {
  if constexpr (N == 0) {
    return 1.0;
  } else if constexpr (N % 2 == 0) {
    const double y = qpow<N / 2>(x);
    return y * y;
  } else {
    return x * qpow<N - 1>(x);
  }
}
constexpr int kQuadGauss = 24;
static __device__ const double kQuadGx[kQuadGauss] = {-0.9951872199970213, -0.9747285559713095, -0.9382745520027328, -0.8864155270044011, -0.820001985973903, -0.7401241915785544, -0.6480936519369755, -0.5454214713888396, -0.4337935076260451, -0.3150426796961634, -0.1911188674736163, -0.06405689286260563, 0.06405689286260563, 0.1911188674736163, 0.3150426796961634, 0.4337935076260451, 0.5454214713888396, 0.6480936519369755, 0.7401241915785544, 0.820001985973903, 0.8864155270044011, 0.9382745520027328, 0.9747285559713095, 0.9951872199970213};
static __device__ const double kQuadGw[kQuadGauss] = {0.01234122979998869, 0.02853138862893356, 0.04427743881741941, 0.05929858491543636, 0.07334648141108016, 0.0861901615319532, 0.09761865210411393, 0.10744427011596556, 0.11550566805372552, 0.1216704729278033, 0.12583745634682825, 0.12793819534675202, 0.12793819534675202, 0.12583745634682825, 0.1216704729278033, 0.11550566805372552, 0.10744427011596556, 0.09761865210411393, 0.0861901615319532, 0.07334648141108016, 0.05929858491543636, 0.04427743881741941, 0.02853138862893356, 0.01234122979998869};
constexpr int kQuadGaussFar = 12;
static __device__ const double kQuadFx[kQuadGaussFar] = {-0.9815606342467192, -0.9041172563704748, -0.7699026741943047, -0.5873179542866175, -0.3678314989981802, -0.1252334085114689, 0.1252334085114689, 0.3678314989981802, 0.5873179542866175, 0.7699026741943047, 0.9041172563704748, 0.9815606342467192};
static __device__ const double kQuadFw[kQuadGaussFar] = {0.04717533638651141, 0.10693932599531907, 0.16007832854334642, 0.20316742672306573, 0.2334925365383546, 0.2491470458134027, 0.2491470458134027, 0.2334925365383546, 0.20316742672306573, 0.16007832854334642, 0.10693932599531907, 0.04717533638651141};
constexpr int kQuadGaussChord = 20;
static __device__ const double kQuadCx[kQuadGaussChord] = {-0.993128599185095, -0.9639719272779138, -0.912234428251326, -0.8391169718222188, -0.7463319064601508, -0.636053680726515, -0.5108670019508271, -0.37370608871541955, -0.22778585114164507, -0.07652652113349734, 0.07652652113349734, 0.22778585114164507, 0.37370608871541955, 0.5108670019508271, 0.636053680726515, 0.7463319064601508, 0.8391169718222188, 0.912234428251326, 0.9639719272779138, 0.993128599185095};
static __device__ const double kQuadCw[kQuadGaussChord] = {0.017614007139150893, 0.040601429800386446, 0.06267204833410879, 0.08327674157670471, 0.1019301198172407, 0.1181945319615186, 0.1316886384491769, 0.1420961093183824, 0.14917298647260424, 0.15275338713072628, 0.15275338713072628, 0.14917298647260424, 0.1420961093183824, 0.1316886384491769, 0.1181945319615186, 0.1019301198172407, 0.08327674157670471, 0.06267204833410879, 0.040601429800386446, 0.017614007139150893};

// ---- w2p5: C2*pi = 621621/16403; pi*W = C u^20 B(u)^5, u = 1 - r, on r <= 1
struct Kern_w2p5 {
  static constexpr int kId = 10;
  static constexpr bool kQuad = true;
  static constexpr int kBlocks = 1;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {1};
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.0;
  __host__ __device__ static __forceinline__ double poly(double r) {
    const double u = 1.0 - r;
    const double b = fma(-4.0, u, 5.0);
    const double b2 = b * b;
    return 37.896787173078096 * qpow<20>(u) * (b2 * b2 * b);
  }
};

// ---- w4p5: C2*pi = 121806372699/2715105619; pi*W = C u^30 B(u)^5, u = 1 - r, on r <= 1
struct Kern_w4p5 {
  static constexpr int kId = 11;
  static constexpr bool kQuad = true;
  static constexpr int kBlocks = 1;
  static constexpr double kR[kBlocks] = {1.0};
  static constexpr int kNA[kBlocks] = {1};
  static constexpr double kMass = 1.0;
  static constexpr double kPlane2 = 0.0;
  __host__ __device__ static __forceinline__ double poly(double r) {
    const double u = 1.0 - r;
    const double b = fma(fma(11.666666666666666, u, -29.333333333333332), u, 18.666666666666668);
    const double b2 = b * b;
    return 44.86248043045283 * qpow<30>(u) * (b2 * b2 * b);
  }
};

// ---- float Chebyshev tables of the block profiles on [0, R] (x = 2 r / R - 1), Clenshaw in float
constexpr int kF32Gauss = 8;   // Gauss-Legendre nodes per panel of the float route
static __device__ const float kF32Gx[kF32Gauss] = {-0.9602898564975362f, -0.7966664774136267f, -0.525532409916329f, -0.18343464249564978f, 0.18343464249564978f, 0.525532409916329f, 0.7966664774136267f, 0.9602898564975362f};
static __device__ const float kF32Gw[kF32Gauss] = {0.10122853629037706f, 0.22238103445337443f, 0.3137066458778869f, 0.36268378337836166f, 0.36268378337836166f, 0.3137066458778869f, 0.22238103445337443f, 0.10122853629037706f};
template <class KT> struct ChebOf;   // the float tables of an exact kernel
struct Cheb_cubic {
  static constexpr double kMhat[] = {0.5714285714285714, -0.07142857142857142};
  static constexpr double kMPhat[] = {-0.04081632653061224, 0.0012755102040816326};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_cubic> : Cheb_cubic {};
template <> __device__ __forceinline__ void Cheb_cubic::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.35714285714285715f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.142857142857143f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.357142857142857f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 3.5714285714285716f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.004464285714285714f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.022321428571428572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.022321428571428572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.08928571428571429f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3125f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.21875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.07142857142857142f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.6428571428571429f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.5f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 2.5f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0006377551020408163f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0047831632653061226f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010841836734693877f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.01403061224489796f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.13392857142857142f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.15401785714285715f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_cubic::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.004464285714285714f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.022321428571428572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.022321428571428572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.08928571428571429f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3125f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.35267857142857145f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -3.985969387755102e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00013950892857142856f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00027901785714285713f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006556919642857143f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.022600446428571428f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.025151466836734693f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_cubic::integrands<1>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.17857142857142858f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.0714285714285714f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.6785714285714284f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, -1.7857142857142858f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0005580357142857143f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0027901785714285715f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0027901785714285715f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.011160714285714286f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0390625f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, 0.02734375f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.03571428571428571f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.32142857142857145f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.25f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, -1.25f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 7.971938775510203e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0005978954081632653f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0013552295918367347f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001753826530612245f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.016741071428571428f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, 0.019252232142857144f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_cubic::potentials<1>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0005580357142857143f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0027901785714285715f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0027901785714285715f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.011160714285714286f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0390625f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, -0.04408482142857143f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.2456154336734693e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.359654017857143e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.719308035714285e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 6.103515625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.103515625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00020490373883928572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0007062639508928571f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, 0.0007859833386479591f - b2);
  }
}
struct Cheb_w2 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.034722222222222224};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_w2> : Cheb_w2 {};
template <> __device__ __forceinline__ void Cheb_w2::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0546875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.2734375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.2734375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.09375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -3.828125f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 2.6796875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.00048828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001708984375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00341796875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02392578125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.02392578125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.080322265625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.27685546875f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.19189453125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0078125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.05859375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1328125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.171875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.640625f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 1.88671875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 5.425347222222222e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0003085666232638889f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.781684027777778e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.004591200086805556f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011406792534722222f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011247422960069444f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.11905924479166667f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.13539632161458334f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_w2::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.00048828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001708984375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00341796875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02392578125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.02392578125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.080322265625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.27685546875f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.30810546875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 3.3908420138888887e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.7220458984375e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.103515625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0001678466796875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.000335693359375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00186920166015625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001495361328125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0060577392578125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019134521484375f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.021711773342556424f - b2);
  }
}
struct Cheb_w4 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.026515151515151516};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_w4> : Cheb_w4 {};
template <> __device__ __forceinline__ void Cheb_w4::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.003204345703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.01904296875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.015380859375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.15380859375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.4844970703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.21533203125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.748291015625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.85009765625f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 3.217620849609375f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 2.002716064453125e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.7738037109375e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0001773834228515625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001590728759765625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0014791488647460938f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0095672607421875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02899932861328125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0112152099609375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.10034751892089844f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.26927947998046875f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.1770153045654297f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0003204345703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.002685546875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0059814453125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.016357421875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.11456298828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.185791015625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3367919921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.199462890625f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 2.2714691162109375f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.6689300537109375e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.1010603471235795e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.2571161443536931e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00019729498660925663f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0005070440696947502f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0008657050855232008f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0068606174353397255f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010787154688979641f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019586288567745323f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.12320899963378906f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.12502527236938477f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_w4::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 2.002716064453125e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.7738037109375e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0001773834228515625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001590728759765625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0014791488647460938f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0095672607421875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02899932861328125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0112152099609375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.10034751892089844f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.26927947998046875f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.3229846954345703f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.043081283569336e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.7093020352450286e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.205371856689453e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 8.304913838704428e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.4513731002807617e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00010788440704345703f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 7.146596908569336e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0006018877029418945f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0015963166952133179f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00041985511779785156f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.005561232566833496f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.014179468154907227f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.017306370265556103f - b2);
  }
}
struct Cheb_w6 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.02142857142857143};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_w6> : Cheb_w6 {};
template <> __device__ __forceinline__ void Cheb_w6::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.00017002650669642856f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0011689322335379465f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0009351457868303571f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.013559613909040178f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.04395185198102679f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.007714952741350446f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.30859810965401785f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.6452505929129464f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.022443498883928572f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.4627064296177457f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.859623500279018f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 3.7492970057896207f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 8.174351283482142e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.317079271589007e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.96999250139509e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 9.431157793317522e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0001018387930733817f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.000752500125340053f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0023670877729143414f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0004821845463344029f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.015108449118477958f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.029658002512795583f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0009935923985072545f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.11313404355730329f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.26185676029750277f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.16634363787514822f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.3078962053571428e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00012138911655970983f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0002795628138950893f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0010667528424944197f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.007101331438337054f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.008967944553920202f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.04006304059709821f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.17900630405970983f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.20514133998325892f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.5587803976876395f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.7741099766322543f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 2.6460268838065013f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 5.4495675223214284e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.0956905909946984e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 3.4059797014508927e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 8.497919355119978e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.4012156895228793e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.825762340000697e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0003787926265171596f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0004723582948957171f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001957314355032785f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.008439732449395316f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.009108775002615793f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.026254715238298688f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.12499693461826869f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.11738677535738264f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_w6::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 8.174351283482142e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.317079271589007e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.96999250139509e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 9.431157793317522e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0001018387930733817f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.000752500125340053f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0023670877729143414f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0004821845463344029f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.015108449118477958f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.029658002512795583f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0009935923985072545f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.11313404355730329f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.26185676029750277f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.3336563621248518f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 3.4059797014508928e-09f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.1974147387913296e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.98276492527553e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 3.9967043059212823e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.37506171635219e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.849504045077733e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 4.732183047703334e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 4.160723515919277e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.000111939651625497f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.729761609009334e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0007122267569814409f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0012720647667135512f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00017956005675452097f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.004980658047965595f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011140206030436925f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.014411726806844985f - b2);
  }
}
struct Cheb_quartic {
  static constexpr double kMhat[] = {0.6515846538782318, -0.15200166805671392, 0.0004170141784820684};
  static constexpr double kMPhat[] = {-0.03490632074347671, 0.0029314607410937687, -8.936018110330037e-07};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_quartic> : Cheb_quartic {};
template <> __device__ __forceinline__ void Cheb_quartic::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.1527151532527106f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.2217212260216848f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 4.276024291075896f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.552048582151793f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 5.345030363844871f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.001590782846382402f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011453636493953295f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.028634091234883235f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.006363131385529608f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.12885341055697455f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.34360909481859886f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.227163790463407f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.025452525542118434f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.28506828607172646f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.445703450792327f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.276024291075896f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 3.7415212546914094f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.00019884785579780026f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0019771158233609855f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.007669845866486581f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010067382870677202f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.028105724075191938f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1574875017918578f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.16011229348838876f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quartic::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.001590782846382402f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011453636493953295f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.028634091234883235f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.006363131385529608f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.12885341055697455f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.34360909481859886f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.4244208634148249f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.2427990987362516e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.385777501061152e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.9654356739340076e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0005965435673934008f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0018791122372892124f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0008351609943507611f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006780711882704988f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.018811007158471903f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.022426842364880833f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quartic::integrands<1>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.09895941930775647f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.7916753544620517f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.7708637406171808f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.5417274812343615f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, -3.4635796757714763f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00037109782240408675f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0026719043213094245f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.006679760803273561f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001484391289616347f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.030058923614731024f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.08015712963928273f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, 0.05299276903930358f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.016493236551292745f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.18472424937447873f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.9368158361134279f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.7708637406171808f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, -2.4245057730400332f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -4.6387227800510844e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00046122157927365063f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0017892216437339896f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0023485190760715773f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006556503312260775f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.03673868441800459f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, 0.03735099582497133f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quartic::potentials<1>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00037109782240408675f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0026719043213094245f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.006679760803273561f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001484391289616347f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.030058923614731024f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.08015712963928273f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, -0.09900889901741035f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.043712625511494e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 6.202635031611164e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.009820602455171e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.009820602455171e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00015780934897733788f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.01374884343724e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0005694496084790711f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0015797634299741972f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, 0.0018834241632765842f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quartic::integrands<2>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0024434424520433694f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019547539616346955f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.06841638865721435f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.1368327773144287f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 0.08552048582151793f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.0181010216847372e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.330327356130108e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.832581839032527e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.072404086738949e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.246618275646372e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00021990982068390325f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.00014538482589658048f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0004072404086738949f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.004561092577147623f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02313125521267723f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.06841638865721435f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 0.059864340075062555f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.2726262771059216e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.2653541269510306e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 4.908701354551412e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.443125037233409e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.7987663408122842e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.000100792001146789f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.0001024718678325688f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quartic::potentials<2>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 1.0181010216847372e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -7.330327356130108e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.832581839032527e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.072404086738949e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.246618275646372e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00021990982068390325f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.0002716293525854879f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 3.181565692764804e-10f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.890759040271655e-09f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.5271515325271059e-09f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.5271515325271058e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.810527327460384e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.1380121455379483e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.735862241972477e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.815617832568808e-07f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -5.741271645409493e-07f - b2);
  }
}
struct Cheb_quintic {
  static constexpr double kMhat[] = {0.7625523012552301, -0.26778242677824265, 0.005230125523012552};
  static constexpr double kMPhat[] = {-0.03177301255230126, 0.004958933829226716, -2.4213544088021077e-05};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_quintic> : Cheb_quintic {};
template <> __device__ __forceinline__ void Cheb_quintic::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0625531184623431f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.6255311846234309f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.814890330805439f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 7.506374215481172f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -13.13615487709205f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 7.88169292625523f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0005585099862709205f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.005212759871861925f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019547849519482217f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.03127655923117155f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.014335089647620293f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.17202107577144352f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3870474204857479f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.24574439395920503f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.008936159780334728f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.11914879707112971f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.7357438219142259f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.764252092050209f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.880843030857741f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 5.5046744246861925f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -6.205666514121339e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.000760194147979864f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.003971626569037657f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.010456548076294456f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.007570913147228034f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.044696313067958945f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1863561654190638f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.17304501074627354f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quintic::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0005585099862709205f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.005212759871861925f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019547849519482217f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.03127655923117155f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.014335089647620293f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.17202107577144352f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3870474204857479f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.5168079072960251f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -3.878541571325837e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 3.1997967963438155e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.144937299784257e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.981374828386506e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0008377649794063807f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001710436832954694f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0069581035789585514f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.01663894334098784f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.02109635724183406f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quintic::integrands<1>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.04942468619246862f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.4942468619246862f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.224110878661088f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.930962343096234f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 10.37918410041841f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, -6.227510460251046f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0001961297071129707f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0018305439330543933f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006864539748953975f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010983263598326359f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.005033995815899582f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.06040794979079498f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.1359178870292887f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, 0.08629707112970711f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.007060669456066946f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.09414225941422594f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.5813284518828452f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.1841004184100417f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.436715481171548f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, -4.349372384937238f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 2.1792189679218967e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00026695432357043235f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001394700139470014f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.003671983960948396f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.002658647140864714f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.015695824616457462f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.06544194560669456f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, 0.06076752092050209f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quintic::potentials<1>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 0.0001961297071129707f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0018305439330543933f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006864539748953975f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010983263598326359f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.005033995815899582f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.06040794979079498f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.1359178870292887f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, -0.18148535564853557f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, 6.053386022005269e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.994043468154347e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.2712110646211065e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.0896094839609484e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0001307531380753138f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00026695432357043235f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0010859774523477453f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0025969026034402603f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, 0.003292587992019216f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quintic::integrands<2>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.003861303608786611f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.03861303608786611f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.1737586623953975f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.4633564330543933f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.8108737578451883f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 0.48652425470711297f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -3.830658342050209e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 3.575281119246862e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00013407304197175733f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0002145168671548117f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 9.83202307792887e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0011798427693514644f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.002654646231040795f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.001685489670502092f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0005516148012552301f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.007354864016736401f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.04541628530334728f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.17063284518828453f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.4247433969665272f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 0.33979471757322177f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -4.2562870467224547e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.213951632235007e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.724023709902371e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 7.171843673727336e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.192670197001395e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0003065590745401848f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0012781630001307532f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.0011868656429785565f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_quintic::potentials<2>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -3.830658342050209e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 3.575281119246862e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00013407304197175733f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0002145168671548117f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 9.83202307792887e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0011798427693514644f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.002654646231040795f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.00354463585251046f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -2.9557548935572604e-09f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 2.4384977871847395e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.207085276470246e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -5.320358808403068e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 6.384430570083682e-07f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.3034879080587518e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 5.302624279041725e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.2680188493360647e-05f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -1.6077089804781327e-05f - b2);
  }
}
struct Cheb_poly6 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.05};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_poly6> : Cheb_poly6 {};
template <> __device__ __forceinline__ void Cheb_poly6::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.001953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0234375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.03515625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.3203125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.158203125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.296875f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 1.87890625f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.52587890625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.000244140625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.003173828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.01324462890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.039306640625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0450439453125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.286376953125f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.2173309326171875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.000244140625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0029296875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00048828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0712890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.058349609375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.818359375f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 1.30908203125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.52587890625e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.44140625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -6.103515625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0006103515625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001373291015625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0110595703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00133056640625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1104736328125f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.15264129638671875f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_poly6::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.52587890625e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.000244140625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.003173828125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.01324462890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.039306640625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0450439453125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.286376953125f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.2826690673828125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -9.5367431640625e-08f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.9073486328125e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -1.049041748046875e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.33514404296875e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00020933151245117188f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.00013580322265625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.002017974853515625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00347137451171875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006358146667480469f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.028347015380859375f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.029538917541503906f - b2);
  }
}
struct Cheb_cone {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.075};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_cone> : Cheb_cone {};
template <> __device__ __forceinline__ void Cheb_cone::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.5f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 1.5f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.03125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.28125f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.25f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.5f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 1.0f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.009375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.09375f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.171875f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_cone::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.03125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.28125f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.25f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.000390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0009765625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.005859375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.04296875f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.0404296875f - b2);
  }
}
struct Cheb_lw2 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.03571428571428571};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_lw2> : Cheb_lw2 {};
template <> __device__ __forceinline__ void Cheb_lw2::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.3125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.6875f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 3.125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.01953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.01953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.078125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.2734375f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.19140625f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.5625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.1875f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 2.1875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0005580357142857143f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.004185267857142857f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.009486607142857142f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.012276785714285714f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1171875f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.134765625f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_lw2::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.01953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.01953125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.078125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.2734375f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.30859375f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -3.487723214285714e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0001220703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.000244140625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.001708984375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.001708984375f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0057373046875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.019775390625f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.022007533482142856f - b2);
  }
}
struct Cheb_lw4 {
  static constexpr double kMhat[] = {0.5};
  static constexpr double kMPhat[] = {-0.027777777777777776};
  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, float& Fl, float& Fp);
  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);
};
template <> struct ChebOf<Kern_lw4> : Cheb_lw4 {};
template <> __device__ __forceinline__ void Cheb_lw4::integrands<0>(float x, float& P, float& Psi, float& Fl, float& Fp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.022786458333333332f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1640625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.41015625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.09114583333333333f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 1.845703125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -4.921875f - b2); b2 = b1; b1 = t;
    P = fmaf(x, b1, 3.25390625f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00017801920572916666f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0010579427083333333f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02691650390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011962890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.09712727864583333f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.2694498697916667f - b2); b2 = b1; b1 = t;
    Psi = fmaf(x, b1, -0.1787567138671875f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.0028483072916666665f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0283203125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.10986328125f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.14420572916666666f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.402587890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -2.255859375f - b2); b2 = b1; b1 = t;
    Fl = fmaf(x, b1, 2.29345703125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.7801920572916668e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.00014919704861111112f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0003323025173611111f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0009087456597222222f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.006364610460069444f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.010321723090277778f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.018710666232638888f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.1221923828125f - b2); b2 = b1; b1 = t;
    Fp = fmaf(x, b1, -0.1261927286783854f - b2);
  }
}
template <> __device__ __forceinline__ void Cheb_lw4::potentials<0>(float x, float& M, float& Mp) {
  const float x2 = 2.0f * x;
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -0.00017801920572916666f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0010579427083333333f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.008544921875f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.02691650390625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.011962890625f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.09712727864583333f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.2694498697916667f - b2); b2 = b1; b1 = t;
    M = fmaf(x, b1, 0.3212432861328125f - b2);
  }
  {
    float b1 = 0.0f, b2 = 0.0f, t;
    t = fmaf(x2, b1, -1.1126200358072917e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 4.874335394965277e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 9.854634602864584e-06f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -8.837381998697917e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 8.217493693033855e-05f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0005315144856770834f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.0016110738118489583f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.0006230672200520834f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, 0.005574862162272136f - b2); b2 = b1; b1 = t;
    t = fmaf(x2, b1, -0.014959971110026041f - b2); b2 = b1; b1 = t;
    Mp = fmaf(x, b1, -0.017943594190809462f - b2);
  }
}

// ---- disk element: pi*W, M/r^2 and the second potential of every exact kernel, summed over its blocks
template <int KID> __device__ __forceinline__ void disk_profile(double r, double ir2, double& P, double& Fl,
                                                             double& F2l);
template <int KID> __device__ __forceinline__ int disk_knots(double* out);
template <> __device__ __forceinline__ void disk_profile<0>(double r, double ir2, double& P, double& Fl, double& F2l) {   // cubic
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(-11.428571428571429, r, 34.285714285714285), r, -34.285714285714285), r, 11.428571428571429);
    Fl += fma(fma(fma(-2.2857142857142856, r, 8.571428571428571), r, -11.428571428571429), r, 5.714285714285714);
    F2l += fma(fma(fma(fma(fma(-0.32653061224489793, r, 1.4285714285714286), r, -2.2857142857142856), r, 1.4285714285714286), r, 0.0), r, -0.2857142857142857);
  } else {
    Fl += 0.5714285714285714 * ir2;
    F2l += -0.04081632653061224 * ir2;
  }
  if (r <= 0.5) {
    P += fma(fma(fma(45.714285714285715, r, -68.57142857142857), r, 34.285714285714285), r, -5.714285714285714);
    Fl += fma(fma(fma(9.142857142857142, r, -17.142857142857142), r, 11.428571428571429), r, -2.857142857142857);
    F2l += fma(fma(fma(fma(fma(1.3061224489795917, r, -2.857142857142857), r, 2.2857142857142856), r, -0.7142857142857143), r, 0.0), r, 0.03571428571428571);
  } else {
    Fl += -0.07142857142857142 * ir2;
    F2l += 0.0012755102040816326 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<0>(double* out) {
  out[0] = 0.5;
  return 1;
}
template <> __device__ __forceinline__ void disk_profile<1>(double r, double ir2, double& P, double& Fl, double& F2l) {   // w2
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(28.0, r, -105.0), r, 140.0), r, -70.0), r, 0.0), r, 7.0);
    Fl += fma(fma(fma(fma(fma(4.0, r, -17.5), r, 28.0), r, -17.5), r, 0.0), r, 3.5);
    F2l += fma(fma(fma(fma(fma(fma(fma(0.4444444444444444, r, -2.1875), r, 4.0), r, -2.9166666666666665), r, 0.0), r, 0.875), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.034722222222222224 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<1>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<2>(double r, double ir2, double& P, double& Fl, double& F2l) {   // w4
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(fma(fma(105.0, r, -576.0), r, 1260.0), r, -1344.0), r, 630.0), r, 0.0), r, -84.0), r, 0.0), r, 9.0);
    Fl += fma(fma(fma(fma(fma(fma(fma(fma(10.5, r, -64.0), r, 157.5), r, -192.0), r, 105.0), r, 0.0), r, -21.0), r, 0.0), r, 4.5);
    F2l += fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(0.875, r, -5.818181818181818), r, 15.75), r, -21.333333333333332), r, 13.125), r, 0.0), r, -3.5), r, 0.0), r, 1.125), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.026515151515151516 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<2>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<3>(double r, double ir2, double& P, double& Fl, double& F2l) {   // w6
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(356.57142857142856, r, -2574.0), r, 7844.571428571428), r, -12870.0), r, 11766.857142857143), r, -5148.0), r, 0.0), r, 735.4285714285714), r, 0.0), r, -122.57142857142857), r, 0.0), r, 11.142857142857142);
    Fl += fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(27.428571428571427, r, -214.5), r, 713.1428571428571), r, -1287.0), r, 1307.4285714285713), r, -643.5), r, 0.0), r, 122.57142857142857), r, 0.0), r, -30.642857142857142), r, 0.0), r, 5.571428571428571);
    F2l += fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.8285714285714285, r, -15.321428571428571), r, 54.857142857142854), r, -107.25), r, 118.85714285714286), r, -64.35), r, 0.0), r, 15.321428571428571), r, 0.0), r, -5.107142857142857), r, 0.0), r, 1.3928571428571428), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.02142857142857143 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<3>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<4>(double r, double ir2, double& P, double& Fl, double& F2l) {   // quartic
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(19.547539616346956, r, -78.19015846538782), r, 117.28523769808173), r, -78.19015846538782), r, 19.547539616346956);
    Fl += fma(fma(fma(fma(3.2579232693911595, r, -15.638031693077565), r, 29.321309424520432), r, -26.063386155129276), r, 9.773769808173478);
    F2l += fma(fma(fma(fma(fma(fma(0.40724040867389494, r, -2.2340045275825093), r, 4.886884904086739), r, -5.212677231025855), r, 2.4434424520433695), r, 0.0), r, -0.3257923269391159);
  } else {
    Fl += 0.6515846538782318 * ir2;
    F2l += -0.03490632074347671 * ir2;
  }
  if (r <= 0.6) {
    P += fma(fma(fma(fma(-97.73769808173478, r, 234.57047539616346), r, -211.11342785654713), r, 84.44537114261885), r, -12.666805671392828);
    Fl += fma(fma(fma(fma(-16.289616346955796, r, 46.914095079232695), r, -52.77835696413678), r, 28.148457047539615), r, -6.333402835696414);
    F2l += fma(fma(fma(fma(fma(fma(-2.0362020433694745, r, 6.702013582747528), r, -8.79639282735613), r, 5.629691409507923), r, -1.5833507089241035), r, 0.0), r, 0.07600083402835696);
  } else {
    Fl += -0.15200166805671392 * ir2;
    F2l += 0.0029314607410937687 * ir2;
  }
  if (r <= 0.2) {
    P += fma(fma(fma(fma(195.47539616346955, r, -156.38031693077565), r, 46.914095079232695), r, -6.255212677231026), r, 0.3127606338615513);
    Fl += fma(fma(fma(fma(32.57923269391159, r, -31.27606338615513), r, 11.728523769808174), r, -2.085070892410342), r, 0.15638031693077564);
    F2l += fma(fma(fma(fma(fma(fma(4.072404086738949, r, -4.468009055165019), r, 1.9547539616346956), r, -0.4170141784820684), r, 0.03909507923269391), r, 0.0), r, -0.0002085070892410342);
  } else {
    Fl += 0.0004170141784820684 * ir2;
    F2l += -8.936018110330037e-07 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<4>(double* out) {
  out[0] = 0.2;
  out[1] = 0.6;
  return 2;
}
template <> __device__ __forceinline__ void disk_profile<5>(double r, double ir2, double& P, double& Fl, double& F2l) {   // quintic
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(-32.02719665271967, r, 160.13598326359832), r, -320.27196652719664), r, 320.27196652719664), r, -160.13598326359832), r, 32.02719665271967);
    Fl += fma(fma(fma(fma(fma(-4.575313807531381, r, 26.689330543933053), r, -64.05439330543933), r, 80.06799163179916), r, -53.37866108786611), r, 16.013598326359833);
    F2l += fma(fma(fma(fma(fma(fma(fma(-0.5083682008368201, r, 3.3361663179916317), r, -9.150627615062762), r, 13.344665271966527), r, -10.675732217573222), r, 4.003399581589958), r, 0.0), r, -0.38127615062761505);
  } else {
    Fl += 0.7625523012552301 * ir2;
    F2l += -0.03177301255230126 * ir2;
  }
  if (r <= 0.6666666666666666) {
    P += fma(fma(fma(fma(fma(192.163179916318, r, -640.5439330543933), r, 854.0585774058577), r, -569.3723849372385), r, 189.7907949790795), r, -25.305439330543933);
    Fl += fma(fma(fma(fma(fma(27.451882845188283, r, -106.75732217573221), r, 170.81171548117155), r, -142.34309623430963), r, 63.26359832635983), r, -12.652719665271967);
    F2l += fma(fma(fma(fma(fma(fma(fma(3.0502092050209204, r, -13.344665271966527), r, 24.401673640167363), r, -23.723849372384937), r, 12.652719665271967), r, -3.1631799163179917), r, 0.0), r, 0.13389121338912133);
  } else {
    Fl += -0.26778242677824265 * ir2;
    F2l += 0.004958933829226716 * ir2;
  }
  if (r <= 0.3333333333333333) {
    P += fma(fma(fma(fma(fma(-480.407949790795, r, 800.6799163179917), r, -533.7866108786611), r, 177.92887029288704), r, -29.65481171548117), r, 1.9769874476987448);
    Fl += fma(fma(fma(fma(fma(-68.6297071129707, r, 133.44665271966528), r, -106.75732217573221), r, 44.48221757322176), r, -9.884937238493723), r, 0.9884937238493724);
    F2l += fma(fma(fma(fma(fma(fma(fma(-7.625523012552302, r, 16.68083158995816), r, -15.251046025104603), r, 7.4137029288702925), r, -1.9769874476987448), r, 0.2471234309623431), r, 0.0), r, -0.002615062761506276);
  } else {
    Fl += 0.005230125523012552 * ir2;
    F2l += -2.4213544088021077e-05 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<5>(double* out) {
  out[0] = 0.3333333333333333;
  out[1] = 0.6666666666666666;
  return 2;
}
template <> __device__ __forceinline__ void disk_profile<6>(double r, double ir2, double& P, double& Fl, double& F2l) {   // poly6
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(-4.0, r, 0.0), r, 12.0), r, 0.0), r, -12.0), r, 0.0), r, 4.0);
    Fl += fma(fma(fma(fma(fma(fma(-0.5, r, 0.0), r, 2.0), r, 0.0), r, -3.0), r, 0.0), r, 2.0);
    F2l += fma(fma(fma(fma(fma(fma(fma(fma(-0.05, r, 0.0), r, 0.25), r, 0.0), r, -0.5), r, 0.0), r, 0.5), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.05 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<6>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<7>(double r, double ir2, double& P, double& Fl, double& F2l) {   // cone
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(-3.0, r, 3.0);
    Fl += fma(-1.0, r, 1.5);
    F2l += fma(fma(fma(-0.2, r, 0.375), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.075 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<7>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<8>(double r, double ir2, double& P, double& Fl, double& F2l) {   // lw2
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(-10.0, r, 30.0), r, -30.0), r, 10.0);
    Fl += fma(fma(fma(-2.0, r, 7.5), r, -10.0), r, 5.0);
    F2l += fma(fma(fma(fma(fma(-0.2857142857142857, r, 1.25), r, -2.0), r, 1.25), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.03571428571428571 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<8>(double* out) {
  return 0;
}
template <> __device__ __forceinline__ void disk_profile<9>(double r, double ir2, double& P, double& Fl, double& F2l) {   // lw4
  P = 0.0;
  Fl = 0.0;
  F2l = 0.25;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(-46.666666666666664, r, 224.0), r, -420.0), r, 373.3333333333333), r, -140.0), r, 0.0), r, 9.333333333333334);
    Fl += fma(fma(fma(fma(fma(fma(-5.833333333333333, r, 32.0), r, -70.0), r, 74.66666666666667), r, -35.0), r, 0.0), r, 4.666666666666667);
    F2l += fma(fma(fma(fma(fma(fma(fma(fma(-0.5833333333333334, r, 3.5555555555555554), r, -8.75), r, 10.666666666666666), r, -5.833333333333333), r, 0.0), r, 1.1666666666666667), r, 0.0), r, -0.25);
  } else {
    Fl += 0.5 * ir2;
    F2l += -0.027777777777777776 * ir2;
  }
}
template <> __device__ __forceinline__ int disk_knots<9>(double* out) {
  return 0;
}
constexpr int kDiskMaxKnots = 2;
// pi*W and its derivative (the far-field rule of the finite-element pair weights)
template <int KID> __device__ __forceinline__ void pi_w_deriv(double r, double& P, double& dP);
template <> __device__ __forceinline__ void pi_w_deriv<0>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(-11.428571428571429, r, 34.285714285714285), r, -34.285714285714285), r, 11.428571428571429);
    dP += fma(fma(-34.285714285714285, r, 68.57142857142857), r, -34.285714285714285);
  }
  if (r <= 0.5) {
    P += fma(fma(fma(45.714285714285715, r, -68.57142857142857), r, 34.285714285714285), r, -5.714285714285714);
    dP += fma(fma(137.14285714285714, r, -137.14285714285714), r, 34.285714285714285);
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<1>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(28.0, r, -105.0), r, 140.0), r, -70.0), r, 0.0), r, 7.0);
    dP += (fma(fma(fma(140.0, r, -420.0), r, 420.0), r, -140.0))*r;
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<2>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(fma(fma(105.0, r, -576.0), r, 1260.0), r, -1344.0), r, 630.0), r, 0.0), r, -84.0), r, 0.0), r, 9.0);
    dP += (fma(fma(fma(fma(fma(fma(840.0, r, -4032.0), r, 7560.0), r, -6720.0), r, 2520.0), r, 0.0), r, -168.0))*r;
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<3>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(356.57142857142856, r, -2574.0), r, 7844.571428571428), r, -12870.0), r, 11766.857142857143), r, -5148.0), r, 0.0), r, 735.4285714285714), r, 0.0), r, -122.57142857142857), r, 0.0), r, 11.142857142857142);
    dP += (fma(fma(fma(fma(fma(fma(fma(fma(fma(3922.285714285714, r, -25740.0), r, 70601.14285714286), r, -102960.0), r, 82368.0), r, -30888.0), r, 0.0), r, 2941.714285714286), r, 0.0), r, -245.14285714285714))*r;
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<4>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(19.547539616346956, r, -78.19015846538782), r, 117.28523769808173), r, -78.19015846538782), r, 19.547539616346956);
    dP += fma(fma(fma(78.19015846538782, r, -234.57047539616346), r, 234.57047539616346), r, -78.19015846538782);
  }
  if (r <= 0.6) {
    P += fma(fma(fma(fma(-97.73769808173478, r, 234.57047539616346), r, -211.11342785654713), r, 84.44537114261885), r, -12.666805671392828);
    dP += fma(fma(fma(-390.9507923269391, r, 703.7114261884905), r, -422.22685571309427), r, 84.44537114261885);
  }
  if (r <= 0.2) {
    P += fma(fma(fma(fma(195.47539616346955, r, -156.38031693077565), r, 46.914095079232695), r, -6.255212677231026), r, 0.3127606338615513);
    dP += fma(fma(fma(781.9015846538782, r, -469.1409507923269), r, 93.82819015846539), r, -6.255212677231026);
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<5>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(-32.02719665271967, r, 160.13598326359832), r, -320.27196652719664), r, 320.27196652719664), r, -160.13598326359832), r, 32.02719665271967);
    dP += fma(fma(fma(fma(-160.13598326359832, r, 640.5439330543933), r, -960.81589958159), r, 640.5439330543933), r, -160.13598326359832);
  }
  if (r <= 0.6666666666666666) {
    P += fma(fma(fma(fma(fma(192.163179916318, r, -640.5439330543933), r, 854.0585774058577), r, -569.3723849372385), r, 189.7907949790795), r, -25.305439330543933);
    dP += fma(fma(fma(fma(960.81589958159, r, -2562.175732217573), r, 2562.175732217573), r, -1138.744769874477), r, 189.7907949790795);
  }
  if (r <= 0.3333333333333333) {
    P += fma(fma(fma(fma(fma(-480.407949790795, r, 800.6799163179917), r, -533.7866108786611), r, 177.92887029288704), r, -29.65481171548117), r, 1.9769874476987448);
    dP += fma(fma(fma(fma(-2402.039748953975, r, 3202.7196652719667), r, -1601.3598326359834), r, 355.8577405857741), r, -29.65481171548117);
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<6>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(-4.0, r, 0.0), r, 12.0), r, 0.0), r, -12.0), r, 0.0), r, 4.0);
    dP += (fma(fma(fma(fma(-24.0, r, 0.0), r, 48.0), r, 0.0), r, -24.0))*r;
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<7>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(-3.0, r, 3.0);
    dP += -3.0;
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<8>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(-10.0, r, 30.0), r, -30.0), r, 10.0);
    dP += fma(fma(-30.0, r, 60.0), r, -30.0);
  }
}
template <> __device__ __forceinline__ void pi_w_deriv<9>(double r, double& P, double& dP) {
  P = 0.0;
  dP = 0.0;
  if (r <= 1.0) {
    P += fma(fma(fma(fma(fma(fma(-46.666666666666664, r, 224.0), r, -420.0), r, 373.3333333333333), r, -140.0), r, 0.0), r, 9.333333333333334);
    dP += (fma(fma(fma(fma(-280.0, r, 1120.0), r, -1680.0), r, 1120.0), r, -280.0))*r;
  }
}
constexpr int kFemGauss = 8;   // nodes per direction of the far-field rule, on [0, 1]
static __device__ const double kFemGx[kFemGauss] = {0.019855071751231912, 0.10166676129318664, 0.2372337950418355, 0.4082826787521751, 0.5917173212478248, 0.7627662049581645, 0.8983332387068134, 0.9801449282487681};
static __device__ const double kFemGw[kFemGauss] = {0.05061426814518853, 0.11119051722668721, 0.15685332293894344, 0.18134189168918083, 0.18134189168918083, 0.15685332293894344, 0.11119051722668721, 0.05061426814518853};

// ---- 3-D radial family (solid half-space / sphere), unit support; W = c3*pi * shape, L = W'/r, dL = L'
template <int K, typename T>
__host__ __device__ __forceinline__ T ipow(T x) {
  T y = x;
#pragma unroll
  for (int i = 1; i < K; ++i) y *= x;
  return y;
}
__host__ __device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__host__ __device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
constexpr int kRadialGauss = 12;
static __device__ const double kRadialGx[kRadialGauss] = {-0.9815606342467192, -0.9041172563704748, -0.7699026741943047, -0.5873179542866175, -0.3678314989981802, -0.1252334085114689, 0.1252334085114689, 0.3678314989981802, 0.5873179542866175, 0.7699026741943047, 0.9041172563704748, 0.9815606342467192};
static __device__ const double kRadialGw[kRadialGauss] = {0.04717533638651141, 0.10693932599531907, 0.16007832854334642, 0.20316742672306573, 0.2334925365383546, 0.2491470458134027, 0.2491470458134027, 0.2334925365383546, 0.20316742672306573, 0.16007832854334642, 0.10693932599531907, 0.04717533638651141};
struct Rad_cubic {   // c3*pi = 16
  static constexpr int kPieces = 2;
  static constexpr double kLo[kPieces] = {0.0, 0.5};
  static constexpr double kHi[kPieces] = {0.5, 1.0};
  template <typename T> __host__ __device__ static __forceinline__ void full(T* v) {
    v[0] = T(1.0); v[1] = T(0.0); v[2] = T(0.075); v[3] = T(0.075); v[4] = T(0.0); v[5] = T(1.0); v[6] = T(1.0); v[7] = T(0.0); v[8] = T(0.0);
  }
  template <int P, typename T> __host__ __device__ static __forceinline__ void eval(T r, T& w, T& l, T& dl);
};
template <> __host__ __device__ __forceinline__ void Rad_cubic::eval<0, double>(double r, double& w, double& l, double& dl) {
  using T = double;
  w = (fma_t((fma_t(T(48.0), r, T(-48.0)) * r), r, T(8.0)));
  l = (fma_t(T(144.0), r, T(-96.0)));
  dl = (T(144.0));
}
template <> __host__ __device__ __forceinline__ void Rad_cubic::eval<0, float>(float r, float& w, float& l, float& dl) {
  using T = float;
  w = (fma_t((fma_t(T(48.0), r, T(-48.0)) * r), r, T(8.0)));
  l = (fma_t(T(144.0), r, T(-96.0)));
  dl = (T(144.0));
}
template <> __host__ __device__ __forceinline__ void Rad_cubic::eval<1, double>(double r, double& w, double& l, double& dl) {
  using T = double;
  w = (T(16.0)) * ipow<3>(T(1.0) - r);
  l = (T(-48.0)) * ipow<2>(T(1.0) - r) * (T(1) / ipow<1>(r));
  dl = (fma_t(T(48.0), r, T(48.0))) * ipow<1>(T(1.0) - r) * (T(1) / ipow<2>(r));
}
template <> __host__ __device__ __forceinline__ void Rad_cubic::eval<1, float>(float r, float& w, float& l, float& dl) {
  using T = float;
  w = (T(16.0)) * ipow<3>(T(1.0) - r);
  l = (T(-48.0)) * ipow<2>(T(1.0) - r) * (T(1) / ipow<1>(r));
  dl = (fma_t(T(48.0), r, T(48.0))) * ipow<1>(T(1.0) - r) * (T(1) / ipow<2>(r));
}
struct Rad_w2 {   // c3*pi = 21/2
  static constexpr int kPieces = 1;
  static constexpr double kLo[kPieces] = {0.0};
  static constexpr double kHi[kPieces] = {1.0};
  template <typename T> __host__ __device__ static __forceinline__ void full(T* v) {
    v[0] = T(1.0); v[1] = T(0.0); v[2] = T(0.06666666666666667); v[3] = T(0.06666666666666667); v[4] = T(0.0); v[5] = T(1.0); v[6] = T(1.0); v[7] = T(0.0); v[8] = T(0.0);
  }
  template <int P, typename T> __host__ __device__ static __forceinline__ void eval(T r, T& w, T& l, T& dl);
};
template <> __host__ __device__ __forceinline__ void Rad_w2::eval<0, double>(double r, double& w, double& l, double& dl) {
  using T = double;
  w = (fma_t(T(42.0), r, T(10.5))) * ipow<4>(T(1.0) - r);
  l = (T(-210.0)) * ipow<3>(T(1.0) - r);
  dl = (T(630.0)) * ipow<2>(T(1.0) - r);
}
template <> __host__ __device__ __forceinline__ void Rad_w2::eval<0, float>(float r, float& w, float& l, float& dl) {
  using T = float;
  w = (fma_t(T(42.0), r, T(10.5))) * ipow<4>(T(1.0) - r);
  l = (T(-210.0)) * ipow<3>(T(1.0) - r);
  dl = (T(630.0)) * ipow<2>(T(1.0) - r);
}
struct Rad_w4 {   // c3*pi = 495/32
  static constexpr int kPieces = 1;
  static constexpr double kLo[kPieces] = {0.0};
  static constexpr double kHi[kPieces] = {1.0};
  template <typename T> __host__ __device__ static __forceinline__ void full(T* v) {
    v[0] = T(1.0); v[1] = T(0.0); v[2] = T(0.05128205128205128); v[3] = T(0.05128205128205128); v[4] = T(0.0); v[5] = T(1.0); v[6] = T(1.0); v[7] = T(0.0); v[8] = T(0.0);
  }
  template <int P, typename T> __host__ __device__ static __forceinline__ void eval(T r, T& w, T& l, T& dl);
};
template <> __host__ __device__ __forceinline__ void Rad_w4::eval<0, double>(double r, double& w, double& l, double& dl) {
  using T = double;
  w = (fma_t(fma_t(T(180.46875), r, T(92.8125)), r, T(15.46875))) * ipow<6>(T(1.0) - r);
  l = (fma_t(T(-1443.75), r, T(-288.75))) * ipow<5>(T(1.0) - r);
  dl = (T(8662.5)) * ipow<4>(T(1.0) - r) * ipow<1>(r);
}
template <> __host__ __device__ __forceinline__ void Rad_w4::eval<0, float>(float r, float& w, float& l, float& dl) {
  using T = float;
  w = (fma_t(fma_t(T(180.46875), r, T(92.8125)), r, T(15.46875))) * ipow<6>(T(1.0) - r);
  l = (fma_t(T(-1443.75), r, T(-288.75))) * ipow<5>(T(1.0) - r);
  dl = (T(8662.5)) * ipow<4>(T(1.0) - r) * ipow<1>(r);
}
struct Rad_w6 {   // c3*pi = 1365/64
  static constexpr int kPieces = 1;
  static constexpr double kLo[kPieces] = {0.0};
  static constexpr double kHi[kPieces] = {1.0};
  template <typename T> __host__ __device__ static __forceinline__ void full(T* v) {
    v[0] = T(1.0); v[1] = T(0.0); v[2] = T(0.041666666666666664); v[3] = T(0.041666666666666664); v[4] = T(0.0); v[5] = T(1.0); v[6] = T(1.0); v[7] = T(0.0); v[8] = T(0.0);
  }
  template <int P, typename T> __host__ __device__ static __forceinline__ void eval(T r, T& w, T& l, T& dl);
};
template <> __host__ __device__ __forceinline__ void Rad_w6::eval<0, double>(double r, double& w, double& l, double& dl) {
  using T = double;
  w = (fma_t(fma_t(fma_t(T(682.5), r, T(533.203125)), r, T(170.625)), r, T(21.328125))) * ipow<8>(T(1.0) - r);
  l = (fma_t(fma_t(T(-7507.5), r, T(-3284.53125)), r, T(-469.21875))) * ipow<7>(T(1.0) - r);
  dl = (fma_t(T(67567.5), r, T(11261.25))) * ipow<6>(T(1.0) - r) * ipow<1>(r);
}
template <> __host__ __device__ __forceinline__ void Rad_w6::eval<0, float>(float r, float& w, float& l, float& dl) {
  using T = float;
  w = (fma_t(fma_t(fma_t(T(682.5), r, T(533.203125)), r, T(170.625)), r, T(21.328125))) * ipow<8>(T(1.0) - r);
  l = (fma_t(fma_t(T(-7507.5), r, T(-3284.53125)), r, T(-469.21875))) * ipow<7>(T(1.0) - r);
  dl = (fma_t(T(67567.5), r, T(11261.25))) * ipow<6>(T(1.0) - r) * ipow<1>(r);
}

// ---- 3-D closed surfaces: compact potentials (unit support, W~ = c3*pi * shape); function ids:
//      0 A_K0, 1 A_K1, 2 A_K2, 3 A_W, 4 A_L, 5 A2_K2
template <class M, int Fn> struct MeshFn;
static __device__ const double kMeshGx8[8] = {-0.9602898564975362, -0.7966664774136267, -0.525532409916329, -0.18343464249564978, 0.18343464249564978, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
static __device__ const double kMeshGw8[8] = {0.10122853629037706, 0.22238103445337443, 0.3137066458778869, 0.36268378337836166, 0.36268378337836166, 0.3137066458778869, 0.22238103445337443, 0.10122853629037706};
struct Mesh_cubic {
  static constexpr int kPieces = 2;
  static constexpr double kBreak = 0.5;   // end of the inner piece
  static constexpr double kQ0 = 0.25, kQ1 = 0.11071428571428571, kQ2 = 0.05625;
};
template <> struct MeshFn<Mesh_cubic, 0> {   // A_K0
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = 0.25;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(1.6, x, -2.4), x, 0.0), x, 1.3333333333333333), x, 0.0), x, -0.7); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.6; dd = b; b = fma(a, b, -2.4); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.3333333333333333); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 5;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.6; b[1] = fma(a, b[0], -2.4); b[2] = fma(a, b[1], 0.0); b[3] = fma(a, b[2], 1.3333333333333333); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
  static constexpr double kNu1 = 0.26666666666666666;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(fma(fma(-0.5333333333333333, x, 2.4), x, -4.0), x, 2.6666666666666665), x, 0.0), x, -0.8); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -0.5333333333333333; dd = b; b = fma(a, b, 2.4); dd = fma(dd, x, b); b = fma(a, b, -4.0); dd = fma(dd, x, b); b = fma(a, b, 2.6666666666666665); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 5;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -0.5333333333333333; b[1] = fma(a, b[0], 2.4); b[2] = fma(a, b[1], -4.0); b[3] = fma(a, b[2], 2.6666666666666665); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
};
template <> struct MeshFn<Mesh_cubic, 1> {   // A_K1
  static constexpr int kNeg = 2;
  static constexpr double kNu0 = 0.055357142857142855;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(1.3714285714285714, x, -2.0), x, 0.0), x, 1.0), x, 0.0), x, -0.35); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.3714285714285714; dd = b; b = fma(a, b, -2.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 5;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.3714285714285714; b[1] = fma(a, b[0], -2.0); b[2] = fma(a, b[1], 0.0); b[3] = fma(a, b[2], 1.0); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
  static constexpr double kNu1 = 0.05714285714285714;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(fma(fma(-0.45714285714285713, x, 2.0), x, -3.2), x, 2.0), x, 0.0), x, -0.4); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -0.45714285714285713; dd = b; b = fma(a, b, 2.0); dd = fma(dd, x, b); b = fma(a, b, -3.2); dd = fma(dd, x, b); b = fma(a, b, 2.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 5;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -0.45714285714285713; b[1] = fma(a, b[0], 2.0); b[2] = fma(a, b[1], -3.2); b[3] = fma(a, b[2], 2.0); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
};
template <> struct MeshFn<Mesh_cubic, 2> {   // A_K2
  static constexpr int kNeg = 3;
  static constexpr double kNu0 = 0.01875;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(1.2, x, -1.7142857142857142), x, 0.0), x, 0.8), x, 0.0), x, -0.23333333333333334); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.2; dd = b; b = fma(a, b, -1.7142857142857142); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 0.8); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 5;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.2; b[1] = fma(a, b[0], -1.7142857142857142); b[2] = fma(a, b[1], 0.0); b[3] = fma(a, b[2], 0.8); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
  static constexpr double kNu1 = 0.01904761904761905;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(fma(fma(-0.4, x, 1.7142857142857142), x, -2.6666666666666665), x, 1.6), x, 0.0), x, -0.26666666666666666); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -0.4; dd = b; b = fma(a, b, 1.7142857142857142); dd = fma(dd, x, b); b = fma(a, b, -2.6666666666666665); dd = fma(dd, x, b); b = fma(a, b, 1.6); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 5;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -0.4; b[1] = fma(a, b[0], 1.7142857142857142); b[2] = fma(a, b[1], -2.6666666666666665); b[3] = fma(a, b[2], 1.6); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
};
template <> struct MeshFn<Mesh_cubic, 3> {   // A_W
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(9.6, x, -12.0), x, 0.0), x, 4.0), x, 0.0), x, -0.7); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 9.6; dd = b; b = fma(a, b, -12.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 4.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 5;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 9.6; b[1] = fma(a, b[0], -12.0); b[2] = fma(a, b[1], 0.0); b[3] = fma(a, b[2], 4.0); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
  static constexpr double kNu1 = 0.0;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(fma(fma(-3.2, x, 12.0), x, -16.0), x, 8.0), x, 0.0), x, -0.8); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -3.2; dd = b; b = fma(a, b, 12.0); dd = fma(dd, x, b); b = fma(a, b, -16.0); dd = fma(dd, x, b); b = fma(a, b, 8.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 5;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -3.2; b[1] = fma(a, b[0], 12.0); b[2] = fma(a, b[1], -16.0); b[3] = fma(a, b[2], 8.0); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
};
template <> struct MeshFn<Mesh_cubic, 4> {   // A_L
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(48.0, x, -48.0), x, 0.0), x, 8.0); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 48.0; dd = b; b = fma(a, b, -48.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 3;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 48.0; b[1] = fma(a, b[0], -48.0); b[2] = fma(a, b[1], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); return dd; }
  static constexpr double kNu1 = 0.0;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(-16.0, x, 48.0), x, -48.0), x, 16.0); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -16.0; dd = b; b = fma(a, b, 48.0); dd = fma(dd, x, b); b = fma(a, b, -48.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 3;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -16.0; b[1] = fma(a, b[0], 48.0); b[2] = fma(a, b[1], -48.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); return dd; }
};
template <> struct MeshFn<Mesh_cubic, 5> {   // A2_K2
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = -0.01875;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(0.17142857142857143, x, -0.2857142857142857), x, 0.0), x, 0.2), x, 0.0), x, -0.11666666666666667), x, 0.0), x, 0.055357142857142855); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.17142857142857143; dd = b; b = fma(a, b, -0.2857142857142857); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 0.2); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.11666666666666667); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 7;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.17142857142857143; b[1] = fma(a, b[0], -0.2857142857142857); b[2] = fma(a, b[1], 0.0); b[3] = fma(a, b[2], 0.2); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], -0.11666666666666667); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
  static constexpr double kNu1 = -0.01904761904761905;
  __host__ __device__ static __forceinline__ double poly1(double x) { return fma(fma(fma(fma(fma(fma(fma(-0.05714285714285714, x, 0.2857142857142857), x, -0.5333333333333333), x, 0.4), x, 0.0), x, -0.13333333333333333), x, 0.0), x, 0.05714285714285714); }
  __host__ __device__ static __forceinline__ double dd1(double x, double a) { double dd; double b = -0.05714285714285714; dd = b; b = fma(a, b, 0.2857142857142857); dd = fma(dd, x, b); b = fma(a, b, -0.5333333333333333); dd = fma(dd, x, b); b = fma(a, b, 0.4); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.13333333333333333); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD1 = 7;
  __host__ __device__ static __forceinline__ void ddb1(double a, double* b) { b[0] = -0.05714285714285714; b[1] = fma(a, b[0], 0.2857142857142857); b[2] = fma(a, b[1], -0.5333333333333333); b[3] = fma(a, b[2], 0.4); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], -0.13333333333333333); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh1(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
};
struct Mesh_w2 {
  static constexpr int kPieces = 1;
  static constexpr double kBreak = 2.0;   // end of the inner piece
  static constexpr double kQ0 = 0.25, kQ1 = 0.10416666666666667, kQ2 = 0.05;
};
template <> struct MeshFn<Mesh_w2, 0> {   // A_K0
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = 0.25;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(0.75, x, -3.75), x, 7.0), x, -5.25), x, 0.0), x, 1.75), x, 0.0), x, -0.75); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.75; dd = b; b = fma(a, b, -3.75); dd = fma(dd, x, b); b = fma(a, b, 7.0); dd = fma(dd, x, b); b = fma(a, b, -5.25); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.75); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 7;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.75; b[1] = fma(a, b[0], -3.75); b[2] = fma(a, b[1], 7.0); b[3] = fma(a, b[2], -5.25); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], 1.75); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
};
template <> struct MeshFn<Mesh_w2, 1> {   // A_K1
  static constexpr int kNeg = 2;
  static constexpr double kNu0 = 0.052083333333333336;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(0.6666666666666666, x, -3.28125), x, 6.0), x, -4.375), x, 0.0), x, 1.3125), x, 0.0), x, -0.375); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.6666666666666666; dd = b; b = fma(a, b, -3.28125); dd = fma(dd, x, b); b = fma(a, b, 6.0); dd = fma(dd, x, b); b = fma(a, b, -4.375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.3125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 7;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.6666666666666666; b[1] = fma(a, b[0], -3.28125); b[2] = fma(a, b[1], 6.0); b[3] = fma(a, b[2], -4.375); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], 1.3125); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
};
template <> struct MeshFn<Mesh_w2, 2> {   // A_K2
  static constexpr int kNeg = 3;
  static constexpr double kNu0 = 0.016666666666666666;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(0.6, x, -2.9166666666666665), x, 5.25), x, -3.75), x, 0.0), x, 1.05), x, 0.0), x, -0.25); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.6; dd = b; b = fma(a, b, -2.9166666666666665); dd = fma(dd, x, b); b = fma(a, b, 5.25); dd = fma(dd, x, b); b = fma(a, b, -3.75); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.05); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 7;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.6; b[1] = fma(a, b[0], -2.9166666666666665); b[2] = fma(a, b[1], 5.25); b[3] = fma(a, b[2], -3.75); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], 1.05); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
};
template <> struct MeshFn<Mesh_w2, 3> {   // A_W
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(6.0, x, -26.25), x, 42.0), x, -26.25), x, 0.0), x, 5.25), x, 0.0), x, -0.75); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 6.0; dd = b; b = fma(a, b, -26.25); dd = fma(dd, x, b); b = fma(a, b, 42.0); dd = fma(dd, x, b); b = fma(a, b, -26.25); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 5.25); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 7;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 6.0; b[1] = fma(a, b[0], -26.25); b[2] = fma(a, b[1], 42.0); b[3] = fma(a, b[2], -26.25); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], 5.25); b[6] = fma(a, b[5], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); return dd; }
};
template <> struct MeshFn<Mesh_w2, 4> {   // A_L
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(42.0, x, -157.5), x, 210.0), x, -105.0), x, 0.0), x, 10.5); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 42.0; dd = b; b = fma(a, b, -157.5); dd = fma(dd, x, b); b = fma(a, b, 210.0); dd = fma(dd, x, b); b = fma(a, b, -105.0); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 5;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 42.0; b[1] = fma(a, b[0], -157.5); b[2] = fma(a, b[1], 210.0); b[3] = fma(a, b[2], -105.0); b[4] = fma(a, b[3], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); return dd; }
};
template <> struct MeshFn<Mesh_w2, 5> {   // A2_K2
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = -0.016666666666666666;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(0.06666666666666667, x, -0.3645833333333333), x, 0.75), x, -0.625), x, 0.0), x, 0.2625), x, 0.0), x, -0.125), x, 0.0), x, 0.052083333333333336); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.06666666666666667; dd = b; b = fma(a, b, -0.3645833333333333); dd = fma(dd, x, b); b = fma(a, b, 0.75); dd = fma(dd, x, b); b = fma(a, b, -0.625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 0.2625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 9;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.06666666666666667; b[1] = fma(a, b[0], -0.3645833333333333); b[2] = fma(a, b[1], 0.75); b[3] = fma(a, b[2], -0.625); b[4] = fma(a, b[3], 0.0); b[5] = fma(a, b[4], 0.2625); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], -0.125); b[8] = fma(a, b[7], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); return dd; }
};
struct Mesh_w4 {
  static constexpr int kPieces = 1;
  static constexpr double kBreak = 2.0;   // end of the inner piece
  static constexpr double kQ0 = 0.25, kQ1 = 0.09114583333333333, kQ2 = 0.038461538461538464;
};
template <> struct MeshFn<Mesh_w4, 0> {   // A_K0
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = 0.25;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.640625, x, -11.0), x, 30.078125), x, -41.25), x, 25.78125), x, 0.0), x, -7.21875), x, 0.0), x, 2.578125), x, 0.0), x, -0.859375); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.640625; dd = b; b = fma(a, b, -11.0); dd = fma(dd, x, b); b = fma(a, b, 30.078125); dd = fma(dd, x, b); b = fma(a, b, -41.25); dd = fma(dd, x, b); b = fma(a, b, 25.78125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -7.21875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 2.578125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 10;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.640625; b[1] = fma(a, b[0], -11.0); b[2] = fma(a, b[1], 30.078125); b[3] = fma(a, b[2], -41.25); b[4] = fma(a, b[3], 25.78125); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -7.21875); b[7] = fma(a, b[6], 0.0); b[8] = fma(a, b[7], 2.578125); b[9] = fma(a, b[8], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); return dd; }
};
template <> struct MeshFn<Mesh_w4, 1> {   // A_K1
  static constexpr int kNeg = 2;
  static constexpr double kNu0 = 0.045572916666666664;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.50390625, x, -10.0), x, 27.0703125), x, -36.666666666666664), x, 22.55859375), x, 0.0), x, -6.015625), x, 0.0), x, 1.93359375), x, 0.0), x, -0.4296875); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.50390625; dd = b; b = fma(a, b, -10.0); dd = fma(dd, x, b); b = fma(a, b, 27.0703125); dd = fma(dd, x, b); b = fma(a, b, -36.666666666666664); dd = fma(dd, x, b); b = fma(a, b, 22.55859375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -6.015625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.93359375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 10;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.50390625; b[1] = fma(a, b[0], -10.0); b[2] = fma(a, b[1], 27.0703125); b[3] = fma(a, b[2], -36.666666666666664); b[4] = fma(a, b[3], 22.55859375); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -6.015625); b[7] = fma(a, b[6], 0.0); b[8] = fma(a, b[7], 1.93359375); b[9] = fma(a, b[8], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); return dd; }
};
template <> struct MeshFn<Mesh_w4, 2> {   // A_K2
  static constexpr int kNeg = 3;
  static constexpr double kNu0 = 0.01282051282051282;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(1.3882211538461537, x, -9.166666666666666), x, 24.609375), x, -33.0), x, 20.052083333333332), x, 0.0), x, -5.15625), x, 0.0), x, 1.546875), x, 0.0), x, -0.2864583333333333); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 1.3882211538461537; dd = b; b = fma(a, b, -9.166666666666666); dd = fma(dd, x, b); b = fma(a, b, 24.609375); dd = fma(dd, x, b); b = fma(a, b, -33.0); dd = fma(dd, x, b); b = fma(a, b, 20.052083333333332); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -5.15625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1.546875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 10;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 1.3882211538461537; b[1] = fma(a, b[0], -9.166666666666666); b[2] = fma(a, b[1], 24.609375); b[3] = fma(a, b[2], -33.0); b[4] = fma(a, b[3], 20.052083333333332); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -5.15625); b[7] = fma(a, b[6], 0.0); b[8] = fma(a, b[7], 1.546875); b[9] = fma(a, b[8], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); return dd; }
};
template <> struct MeshFn<Mesh_w4, 3> {   // A_W
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(18.046875, x, -110.0), x, 270.703125), x, -330.0), x, 180.46875), x, 0.0), x, -36.09375), x, 0.0), x, 7.734375), x, 0.0), x, -0.859375); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 18.046875; dd = b; b = fma(a, b, -110.0); dd = fma(dd, x, b); b = fma(a, b, 270.703125); dd = fma(dd, x, b); b = fma(a, b, -330.0); dd = fma(dd, x, b); b = fma(a, b, 180.46875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -36.09375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 7.734375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 10;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 18.046875; b[1] = fma(a, b[0], -110.0); b[2] = fma(a, b[1], 270.703125); b[3] = fma(a, b[2], -330.0); b[4] = fma(a, b[3], 180.46875); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -36.09375); b[7] = fma(a, b[6], 0.0); b[8] = fma(a, b[7], 7.734375); b[9] = fma(a, b[8], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); return dd; }
};
template <> struct MeshFn<Mesh_w4, 4> {   // A_L
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(180.46875, x, -990.0), x, 2165.625), x, -2310.0), x, 1082.8125), x, 0.0), x, -144.375), x, 0.0), x, 15.46875); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 180.46875; dd = b; b = fma(a, b, -990.0); dd = fma(dd, x, b); b = fma(a, b, 2165.625); dd = fma(dd, x, b); b = fma(a, b, -2310.0); dd = fma(dd, x, b); b = fma(a, b, 1082.8125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -144.375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 8;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 180.46875; b[1] = fma(a, b[0], -990.0); b[2] = fma(a, b[1], 2165.625); b[3] = fma(a, b[2], -2310.0); b[4] = fma(a, b[3], 1082.8125); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -144.375); b[7] = fma(a, b[6], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); return dd; }
};
template <> struct MeshFn<Mesh_w4, 5> {   // A2_K2
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = -0.01282051282051282;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(0.11568509615384616, x, -0.8333333333333334), x, 2.4609375), x, -3.6666666666666665), x, 2.5065104166666665), x, 0.0), x, -0.859375), x, 0.0), x, 0.38671875), x, 0.0), x, -0.14322916666666666), x, 0.0), x, 0.045572916666666664); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.11568509615384616; dd = b; b = fma(a, b, -0.8333333333333334); dd = fma(dd, x, b); b = fma(a, b, 2.4609375); dd = fma(dd, x, b); b = fma(a, b, -3.6666666666666665); dd = fma(dd, x, b); b = fma(a, b, 2.5065104166666665); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.859375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 0.38671875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.14322916666666666); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 12;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.11568509615384616; b[1] = fma(a, b[0], -0.8333333333333334); b[2] = fma(a, b[1], 2.4609375); b[3] = fma(a, b[2], -3.6666666666666665); b[4] = fma(a, b[3], 2.5065104166666665); b[5] = fma(a, b[4], 0.0); b[6] = fma(a, b[5], -0.859375); b[7] = fma(a, b[6], 0.0); b[8] = fma(a, b[7], 0.38671875); b[9] = fma(a, b[8], 0.0); b[10] = fma(a, b[9], -0.14322916666666666); b[11] = fma(a, b[10], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); return dd; }
};
struct Mesh_w6 {
  static constexpr int kPieces = 1;
  static constexpr double kBreak = 2.0;   // end of the inner piece
  static constexpr double kQ0 = 0.25, kQ1 = 0.08203125, kQ2 = 0.03125;
};
template <> struct MeshFn<Mesh_w6, 0> {   // A_K0
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = 0.25;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(3.75, x, -31.58203125), x, 113.75), x, -223.9453125), x, 250.25), x, -136.85546875), x, 0.0), x, 33.515625), x, 0.0), x, -11.73046875), x, 0.0), x, 3.5546875), x, 0.0), x, -0.95703125); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 3.75; dd = b; b = fma(a, b, -31.58203125); dd = fma(dd, x, b); b = fma(a, b, 113.75); dd = fma(dd, x, b); b = fma(a, b, -223.9453125); dd = fma(dd, x, b); b = fma(a, b, 250.25); dd = fma(dd, x, b); b = fma(a, b, -136.85546875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 33.515625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -11.73046875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 3.5546875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 13;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 3.75; b[1] = fma(a, b[0], -31.58203125); b[2] = fma(a, b[1], 113.75); b[3] = fma(a, b[2], -223.9453125); b[4] = fma(a, b[3], 250.25); b[5] = fma(a, b[4], -136.85546875); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 33.515625); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -11.73046875); b[10] = fma(a, b[9], 0.0); b[11] = fma(a, b[10], 3.5546875); b[12] = fma(a, b[11], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); dd = fma(dd, x, b[12]); return dd; }
};
template <> struct MeshFn<Mesh_w6, 1> {   // A_K1
  static constexpr int kNeg = 2;
  static constexpr double kNu0 = 0.041015625;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(3.5, x, -29.326171875), x, 105.0), x, -205.283203125), x, 227.5), x, -123.169921875), x, 0.0), x, 29.326171875), x, 0.0), x, -9.775390625), x, 0.0), x, 2.666015625), x, 0.0), x, -0.478515625); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 3.5; dd = b; b = fma(a, b, -29.326171875); dd = fma(dd, x, b); b = fma(a, b, 105.0); dd = fma(dd, x, b); b = fma(a, b, -205.283203125); dd = fma(dd, x, b); b = fma(a, b, 227.5); dd = fma(dd, x, b); b = fma(a, b, -123.169921875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 29.326171875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -9.775390625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 2.666015625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 13;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 3.5; b[1] = fma(a, b[0], -29.326171875); b[2] = fma(a, b[1], 105.0); b[3] = fma(a, b[2], -205.283203125); b[4] = fma(a, b[3], 227.5); b[5] = fma(a, b[4], -123.169921875); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 29.326171875); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -9.775390625); b[10] = fma(a, b[9], 0.0); b[11] = fma(a, b[10], 2.666015625); b[12] = fma(a, b[11], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); dd = fma(dd, x, b[12]); return dd; }
};
template <> struct MeshFn<Mesh_w6, 2> {   // A_K2
  static constexpr int kNeg = 3;
  static constexpr double kNu0 = 0.010416666666666666;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(3.28125, x, -27.37109375), x, 97.5), x, -189.4921875), x, 208.54166666666666), x, -111.97265625), x, 0.0), x, 26.067708333333332), x, 0.0), x, -8.37890625), x, 0.0), x, 2.1328125), x, 0.0), x, -0.3190104166666667); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 3.28125; dd = b; b = fma(a, b, -27.37109375); dd = fma(dd, x, b); b = fma(a, b, 97.5); dd = fma(dd, x, b); b = fma(a, b, -189.4921875); dd = fma(dd, x, b); b = fma(a, b, 208.54166666666666); dd = fma(dd, x, b); b = fma(a, b, -111.97265625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 26.067708333333332); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -8.37890625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 2.1328125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 13;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 3.28125; b[1] = fma(a, b[0], -27.37109375); b[2] = fma(a, b[1], 97.5); b[3] = fma(a, b[2], -189.4921875); b[4] = fma(a, b[3], 208.54166666666666); b[5] = fma(a, b[4], -111.97265625); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 26.067708333333332); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -8.37890625); b[10] = fma(a, b[9], 0.0); b[11] = fma(a, b[10], 2.1328125); b[12] = fma(a, b[11], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); dd = fma(dd, x, b[12]); return dd; }
};
template <> struct MeshFn<Mesh_w6, 3> {   // A_W
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(52.5, x, -410.56640625), x, 1365.0), x, -2463.3984375), x, 2502.5), x, -1231.69921875), x, 0.0), x, 234.609375), x, 0.0), x, -58.65234375), x, 0.0), x, 10.6640625), x, 0.0), x, -0.95703125); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 52.5; dd = b; b = fma(a, b, -410.56640625); dd = fma(dd, x, b); b = fma(a, b, 1365.0); dd = fma(dd, x, b); b = fma(a, b, -2463.3984375); dd = fma(dd, x, b); b = fma(a, b, 2502.5); dd = fma(dd, x, b); b = fma(a, b, -1231.69921875); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 234.609375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -58.65234375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 10.6640625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 13;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 52.5; b[1] = fma(a, b[0], -410.56640625); b[2] = fma(a, b[1], 1365.0); b[3] = fma(a, b[2], -2463.3984375); b[4] = fma(a, b[3], 2502.5); b[5] = fma(a, b[4], -1231.69921875); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 234.609375); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -58.65234375); b[10] = fma(a, b[9], 0.0); b[11] = fma(a, b[10], 10.6640625); b[12] = fma(a, b[11], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); dd = fma(dd, x, b[12]); return dd; }
};
template <> struct MeshFn<Mesh_w6, 4> {   // A_L
  static constexpr int kNeg = 0;
  static constexpr double kNu0 = 0.0;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(682.5, x, -4926.796875), x, 15015.0), x, -24633.984375), x, 22522.5), x, -9853.59375), x, 0.0), x, 1407.65625), x, 0.0), x, -234.609375), x, 0.0), x, 21.328125); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 682.5; dd = b; b = fma(a, b, -4926.796875); dd = fma(dd, x, b); b = fma(a, b, 15015.0); dd = fma(dd, x, b); b = fma(a, b, -24633.984375); dd = fma(dd, x, b); b = fma(a, b, 22522.5); dd = fma(dd, x, b); b = fma(a, b, -9853.59375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 1407.65625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -234.609375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 11;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 682.5; b[1] = fma(a, b[0], -4926.796875); b[2] = fma(a, b[1], 15015.0); b[3] = fma(a, b[2], -24633.984375); b[4] = fma(a, b[3], 22522.5); b[5] = fma(a, b[4], -9853.59375); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 1407.65625); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -234.609375); b[10] = fma(a, b[9], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); return dd; }
};
template <> struct MeshFn<Mesh_w6, 5> {   // A2_K2
  static constexpr int kNeg = 1;
  static constexpr double kNu0 = -0.010416666666666666;
  __host__ __device__ static __forceinline__ double poly0(double x) { return fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(fma(0.21875, x, -1.955078125), x, 7.5), x, -15.791015625), x, 18.958333333333332), x, -11.197265625), x, 0.0), x, 3.2584635416666665), x, 0.0), x, -1.396484375), x, 0.0), x, 0.533203125), x, 0.0), x, -0.15950520833333334), x, 0.0), x, 0.041015625); }
  __host__ __device__ static __forceinline__ double dd0(double x, double a) { double dd; double b = 0.21875; dd = b; b = fma(a, b, -1.955078125); dd = fma(dd, x, b); b = fma(a, b, 7.5); dd = fma(dd, x, b); b = fma(a, b, -15.791015625); dd = fma(dd, x, b); b = fma(a, b, 18.958333333333332); dd = fma(dd, x, b); b = fma(a, b, -11.197265625); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 3.2584635416666665); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -1.396484375); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, 0.533203125); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); b = fma(a, b, -0.15950520833333334); dd = fma(dd, x, b); b = fma(a, b, 0.0); dd = fma(dd, x, b); return dd; }
  static constexpr int kDD0 = 15;
  __host__ __device__ static __forceinline__ void ddb0(double a, double* b) { b[0] = 0.21875; b[1] = fma(a, b[0], -1.955078125); b[2] = fma(a, b[1], 7.5); b[3] = fma(a, b[2], -15.791015625); b[4] = fma(a, b[3], 18.958333333333332); b[5] = fma(a, b[4], -11.197265625); b[6] = fma(a, b[5], 0.0); b[7] = fma(a, b[6], 3.2584635416666665); b[8] = fma(a, b[7], 0.0); b[9] = fma(a, b[8], -1.396484375); b[10] = fma(a, b[9], 0.0); b[11] = fma(a, b[10], 0.533203125); b[12] = fma(a, b[11], 0.0); b[13] = fma(a, b[12], -0.15950520833333334); b[14] = fma(a, b[13], 0.0); }
  __host__ __device__ static __forceinline__ double ddh0(double x, const double* b) { double dd = b[0]; dd = fma(dd, x, b[1]); dd = fma(dd, x, b[2]); dd = fma(dd, x, b[3]); dd = fma(dd, x, b[4]); dd = fma(dd, x, b[5]); dd = fma(dd, x, b[6]); dd = fma(dd, x, b[7]); dd = fma(dd, x, b[8]); dd = fma(dd, x, b[9]); dd = fma(dd, x, b[10]); dd = fma(dd, x, b[11]); dd = fma(dd, x, b[12]); dd = fma(dd, x, b[13]); dd = fma(dd, x, b[14]); return dd; }
};

// ---- 2-D conditioned triangles: pi W and rho = -pi W'/r per piece (unit support)
static __device__ const double kTriGx16[16] = {-0.9894009349916499, -0.9445750230732326, -0.8656312023878318, -0.755404408355003, -0.6178762444026438, -0.45801677765722737, -0.2816035507792589, -0.09501250983763744, 0.09501250983763744, 0.2816035507792589, 0.45801677765722737, 0.6178762444026438, 0.755404408355003, 0.8656312023878318, 0.9445750230732326, 0.9894009349916499};
static __device__ const double kTriGw16[16] = {0.027152459411754176, 0.062253523938647456, 0.0951585116824926, 0.12462897125553407, 0.1495959888165767, 0.16915651939500265, 0.18260341504492364, 0.18945061045506864, 0.18945061045506864, 0.18260341504492364, 0.16915651939500265, 0.1495959888165767, 0.12462897125553407, 0.0951585116824926, 0.062253523938647456, 0.027152459411754176};
static __device__ const double kTriGx8[8] = {-0.9602898564975362, -0.7966664774136267, -0.525532409916329, -0.18343464249564978, 0.18343464249564978, 0.525532409916329, 0.7966664774136267, 0.9602898564975362};
static __device__ const double kTriGw8[8] = {0.10122853629037706, 0.22238103445337443, 0.3137066458778869, 0.36268378337836166, 0.36268378337836166, 0.3137066458778869, 0.22238103445337443, 0.10122853629037706};
struct Tri_cubic {
  static constexpr int kPieces = 2;
  static constexpr double kPlane2 = 0.07908163265306123;   // int_plane y_x^2 W
  static constexpr double kKnot = 0.5;   // end of the inner piece
  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);
};
template <> __host__ __device__ __forceinline__ void Tri_cubic::eval<0>(double r, double& w, double& rho) {
  using T = double;
  w = (fma_t((fma_t(T(34.285714285714285), r, T(-34.285714285714285)) * r), r, T(5.714285714285714)));
  rho = (fma_t(T(-102.85714285714286), r, T(68.57142857142857)));
}
template <> __host__ __device__ __forceinline__ void Tri_cubic::eval<1>(double r, double& w, double& rho) {
  using T = double;
  w = (T(11.428571428571429)) * ipow<3>(T(1.0) - r);
  rho = (T(34.285714285714285)) * ipow<2>(T(1.0) - r) * (T(1) / ipow<1>(r));
}
struct Tri_w2 {
  static constexpr int kPieces = 1;
  static constexpr double kPlane2 = 0.06944444444444445;   // int_plane y_x^2 W
  static constexpr double kKnot = 2.0;   // end of the inner piece
  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);
};
template <> __host__ __device__ __forceinline__ void Tri_w2::eval<0>(double r, double& w, double& rho) {
  using T = double;
  w = (fma_t(T(28.0), r, T(7.0))) * ipow<4>(T(1.0) - r);
  rho = (T(140.0)) * ipow<3>(T(1.0) - r);
}
struct Tri_w4 {
  static constexpr int kPieces = 1;
  static constexpr double kPlane2 = 0.05303030303030303;   // int_plane y_x^2 W
  static constexpr double kKnot = 2.0;   // end of the inner piece
  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);
};
template <> __host__ __device__ __forceinline__ void Tri_w4::eval<0>(double r, double& w, double& rho) {
  using T = double;
  w = (fma_t(fma_t(T(105.0), r, T(54.0)), r, T(9.0))) * ipow<6>(T(1.0) - r);
  rho = (fma_t(T(840.0), r, T(168.0))) * ipow<5>(T(1.0) - r);
}
struct Tri_w6 {
  static constexpr int kPieces = 1;
  static constexpr double kPlane2 = 0.04285714285714286;   // int_plane y_x^2 W
  static constexpr double kKnot = 2.0;   // end of the inner piece
  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);
};
template <> __host__ __device__ __forceinline__ void Tri_w6::eval<0>(double r, double& w, double& rho) {
  using T = double;
  w = (fma_t(fma_t(fma_t(T(356.57142857142856), r, T(278.57142857142856)), r, T(89.14285714285714)), r, T(11.142857142857142))) * ipow<8>(T(1.0) - r);
  rho = (fma_t(fma_t(T(3922.285714285714), r, T(1716.0)), r, T(245.14285714285714))) * ipow<7>(T(1.0) - r);
}
struct Tri_poly6 {
  static constexpr int kPieces = 1;
  static constexpr double kPlane2 = 0.1;   // int_plane y_x^2 W
  static constexpr double kKnot = 2.0;   // end of the inner piece
  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);
};
template <> __host__ __device__ __forceinline__ void Tri_poly6::eval<0>(double r, double& w, double& rho) {
  using T = double;
  w = (fma_t(fma_t(fma_t(T(4.0), r, T(12.0)), r, T(12.0)), r, T(4.0))) * ipow<3>(T(1.0) - r);
  rho = (fma_t(fma_t(T(24.0), r, T(48.0)), r, T(24.0))) * ipow<2>(T(1.0) - r);
}

}  // namespace wsb
