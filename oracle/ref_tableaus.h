// Generated by oracle/gen_ref_tableaus.py from tests/golden/ref_tableaus.json
// (the reference's odesolve/tableau/*.rs, evaluated bit for bit). Oracle only.
#pragma once

// dopri5: 7 stages; a is s x s row-major, rows zero-padded
static const double ref_dopri5_c[7] = {0.0, 0x1.999999999999ap-3, 0x1.3333333333333p-2, 0x1.999999999999ap-1, 0x1.c71c71c71c71cp-1, 0x1.0000000000000p+0, 0x1.0000000000000p+0};
static const double ref_dopri5_a[49] = {
  0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.999999999999ap-3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.3333333333333p-4, 0x1.ccccccccccccdp-3, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.f49f49f49f49fp-1, -0x1.ddddddddddddep+1, 0x1.c71c71c71c71cp+1, 0.0, 0.0, 0.0, 0.0,
  0x1.79eec0fc37181p+1, -0x1.7310bd29520e4p+3, 0x1.3a552363c5290p+3, -0x1.29c9eba1e3345p-2, 0.0, 0.0, 0.0,
  0x1.6c52bf5a814b0p+1, -0x1.583e0f83e0f84p+3, 0x1.1d016a3721e8bp+3, 0x1.1d1745d1745d1p-2, -0x1.1818970d9cc2fp-2, 0.0, 0.0,
  0x1.7555555555555p-4, 0.0, 0x1.cc0499a5605fbp-2, 0x1.4d55555555555p-1, -0x1.4a1cfb2b78c13p-2, 0x1.0c30c30c30c31p-3, 0.0,
};
static const double ref_dopri5_b[7] = {0x1.7555555555555p-4, 0.0, 0x1.cc0499a5605fbp-2, 0x1.4d55555555555p-1, -0x1.4a1cfb2b78c13p-2, 0x1.0c30c30c30c31p-3, 0.0};
static const double ref_dopri5_e[7] = {0x1.4320fedcba980p-10, 0.0, -0x1.16b5a550abfc0p-8, 0x1.2eeeeeeeeeef0p-5, -0x1.a0ad1d2ca1858p-5, 0x1.5748a7bdaf0e4p-5, -0x1.999999999999ap-6};

// dop853: 12 stages; a is s x s row-major, rows zero-padded
static const double ref_dop853_c[12] = {0.0, 0x1.aee6838dae63ap-5, 0x1.432ce2aa42cacp-4, 0x1.e4c353ff64302p-4, 0x1.2068c499c08d9p-2, 0x1.5555555555555p-2, 0x1.0000000000000p-2, 0x1.3b13b13b13b14p-2, 0x1.4d74d74d74d75p-1, 0x1.3333333333333p-1, 0x1.b6db6db6db6dbp-1, 0x1.0000000000000p+0};
static const double ref_dop853_a[144] = {
  0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.aee6838dae63ap-5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.432ce2aa42cacp-6, 0x1.e4c353ff64302p-5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.e4c353ff64302p-6, 0.0, 0x1.6b927eff8b241p-4, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.ee50d7ecde9fap-3, 0.0, -0x1.c4e3ab5ad1507p-1, 0x1.d983d7ac79ef5p-1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.2f684bda12f68p-5, 0.0, 0.0, 0x1.5ddb63bdb6d36p-3, 0x1.00f533f66f19ap-3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.3000000000000p-5, 0.0, 0.0, 0x1.5cad30f3347edp-3, 0x1.ed4b3c332e04dp-5, -0x1.2000000000000p-6, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.2fdb8fee78792p-5, 0.0, 0.0, 0x1.5cf23f6595d72p-3, 0x1.b758640dea698p-4, -0x1.f5fcc20fcd32fp-7, 0x1.0f1d92efb0b71p-7, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.3f8b78b985813p-1, 0.0, 0.0, -0x1.ae31bacc6bc8ap+1, -0x1.bc873f08e11f9p-1, 0x1.b9793d88d1855p+4, 0x1.42770f892ad69p+4, -0x1.5beb4865c42f9p+5, 0.0, 0.0, 0.0, 0.0,
  0x1.e9205e321b655p-2, 0.0, 0.0, -0x1.3e7a8a34bd27fp+1, -0x1.2e3a9968c93c8p-1, 0x1.53ae4a6d655eep+4, 0x1.e8ef7b5f258b8p+3, -0x1.0a4e418d711b9p+5, -0x1.4d1b3d9b4a876p-6, 0.0, 0.0, 0.0,
  -0x1.dfd121f1d399bp-1, 0.0, 0.0, 0x1.4bed869fb0b9dp+2, 0x1.1768702792ea9p+0, -0x1.04cb0e2110c1cp+3, -0x1.2852305e975a8p+4, 0x1.6bd4f06cb863ap+4, 0x1.3f2e777cf109dp+1, -0x1.85fc60d2b572cp+1, 0.0, 0.0,
  0x1.22fbd3b09fcdcp+1, 0.0, 0.0, -0x1.511a963cafe55p+3, -0x1.001c935ac72acp+1, -0x1.1f57c8eff3006p+4, 0x1.bf2ea18b58a01p+4, -0x1.6df3a7d1cec13p+1, -0x1.1bee71a9f33a9p+3, 0x1.8b89c42c81861p+3, 0x1.496ac6253e202p-1, 0.0,
};
static const double ref_dop853_b[12] = {0x1.bcc6368d1177cp-5, 0.0, 0.0, 0.0, 0.0, 0x1.1cd1ed2ad5ae2p+2, 0x1.e43a845d5ab9fp+0, -0x1.7346ecf96af43p+2, 0x1.3ea1df2f0eb98p-2, -0x1.37a028f43b002p-3, 0x1.9c657697fe72dp-3, 0x1.6e44f50ab6bc2p-5};
static const double ref_dop853_e[12] = {0x1.adeaea1607e1ap-7, 0.0, 0.0, 0.0, 0.0, -0x1.39a3da55ab5c3p+0, -0x1.fba83bede8a72p-2, 0x1.aa149f7eda509p+0, -0x1.66bc9b10e7e71p-2, 0x1.56330d0783989p-2, 0x1.4f8eb54a31435p-4, -0x1.6e44f50ab6bc2p-6};
static const double ref_dop853_e3[12] = {-0x1.84b641fbfa1f1p-3, 0.0, 0.0, 0.0, 0.0, 0x1.1cd1ed2ad5ae2p+2, 0x1.e43a845d5ab9fp+0, -0x1.7346ecf96af43p+2, -0x1.b0d3a26abb716p-2, -0x1.37a028f43b002p-3, 0x1.9c657697fe72dp-3, 0x1.732080ac040edp-6};

// vern7: 10 stages; a is s x s row-major, rows zero-padded
static const double ref_vern7_c[10] = {0.0, 0x1.47ae147ae147bp-8, 0x1.be02468acf135p-4, 0x1.4e81b4e81b4e8p-3, 0x1.d26e978d4fdf4p-2, 0x1.38119f5c18ee8p-1, 0x1.c49ba5e353f7dp-1, 0x1.d99999999999ap-1, 0x1.0000000000000p+0, 0x1.0000000000000p+0};
static const double ref_vern7_a[100] = {
  0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.47ae147ae147bp-8, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  -0x1.13a8847ce7186p+0, 0x1.2f88a8e59409ap+0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.4e81b4e81b4e8p-5, 0.0, 0x1.f5c28f5c28f5cp-4, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.471fb9cddc9bdp-1, 0.0, -0x1.3a537b236d238p+1, 0x1.22d95fa19ff87p+1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  -0x1.54ae9142bd52dp+1, 0.0, 0x1.59be93e7f0391p+3, -0x1.0b5344d4e2ef6p+3, 0x1.a416f336399e6p-1, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.8455e02ba6d51p+2, 0.0, -0x1.8b616076cbec1p+4, 0x1.46d71d0ab3120p+4, -0x1.e7f9f82406e6ep+0, 0x1.01948128a32f7p+0, 0.0, 0.0, 0.0, 0.0,
  0x1.81bfdb75b2798p+3, 0.0, -0x1.8e09ccb12e37ep+5, 0x1.4924a2cc6e376p+5, -0x1.1d8d7a71af007p+2, 0x1.056b3a3a7fe6cp+1, -0x1.92d5cf70abb44p-4, 0.0, 0.0, 0.0,
  0x1.446bb241baabep+3, 0.0, -0x1.55210bed841c7p+5, 0x1.1e1c582ab6be0p+5, -0x1.164601976fe88p+2, 0x1.01432ab412663p+1, 0x1.651e784ce7ec1p-2, -0x1.15f41b4722d81p-2, 0.0, 0.0,
  -0x1.683d96681eb23p+5, 0.0, 0x1.76a78c7eacee8p+7, -0x1.340ec1faa9e18p+7, 0x1.2908d1a693680p+4, -0x1.c91368e7b5080p+2, 0x1.4f0e1437ed68ep+0, 0.0, 0.0, 0.0,
};
static const double ref_vern7_b[10] = {0x1.824c7fe71401bp-5, 0.0, 0.0, 0x1.07af8f2c9ce02p-2, 0x1.0c7562a9bdcddp-2, 0x1.37a025dab0159p-3, 0x1.f9da53eb6a44fp-2, -0x1.2d5dcbdcea09dp-2, 0x1.4d138cc3aa307p-4, 0.0};
static const double ref_vern7_e[10] = {0x1.4dd7897422b5dp-9, 0.0, 0.0, -0x1.3c7c7d0e25406p-7, 0x1.5898171705ca6p-5, -0x1.11216681df170p-4, 0x1.0f5eb708b4517p-2, -0x1.2d5dcbdcea09dp-2, 0x1.4d138cc3aa307p-4, -0x1.4c842c994e2b0p-6};

// vern9: 16 stages; a is s x s row-major, rows zero-padded
static const double ref_vern9_c[16] = {0.0, 0x1.1b9b66f9335d2p-5, 0x1.8d6967ce8c140p-4, 0x1.2a0f0ddae90f0p-3, 0x1.1f3b645a1cac1p-1, 0x1.d5021996737dfp-3, 0x1.170933f898600p-1, 0x1.4a3d70a3d70a4p-1, 0x1.ef5c28f5c28f6p-2, 0x1.14c447c30d307p-4, 0x1.0000000000000p-2, 0x1.5170f9cd5cc3bp-1, 0x1.a425aee631f8ap-1, 0x1.cd6a161e4f766p-1, 0x1.0000000000000p+0, 0x1.0000000000000p+0};
static const double ref_vern9_a[256] = {
  0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.1b9b66f9335d2p-5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  -0x1.3ef18f369c59bp-5, 0x1.167117b4ed206p-3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.2a0f0ddae90f0p-5, 0.0, 0x1.bf1694c85d968p-4, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.034c3b60de98fp+1, 0.0, -0x1.e8d561edf47b4p+2, 0x1.8b16b0c8c8c45p+2, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.a2cc3094af286p-5, 0.0, 0.0, 0x1.6aaa2aa3ac883p-3, 0x1.a4e2cd9b2bacap-11, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.0d84a25710b76p-3, 0.0, 0.0, -0x1.2ed338fc2e70cp-2, 0x1.67af6c2c4dcabp-4, 0x1.3e1bba5b61b13p-1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.258bf258bf259p-4, 0.0, 0.0, 0.0, 0.0, 0x1.527c9456e8906p-2, 0x1.f136a0b52b758p-3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.261eb851eb852p-4, 0.0, 0.0, 0.0, 0.0, 0x1.515833d6d2263p-2, 0x1.dd4307aef4d7fp-4, -0x1.16a3d70a3d70ap-5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.8c3a28e31b86ap-5, 0.0, 0.0, 0.0, 0.0, 0x1.41dce40bdea02p-5, 0x1.b0059aad5ca01p-4, -0x1.5f403a3623eb5p-6, -0x1.aa7ccad443883p-4, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  -0x1.b48fcf1d415e2p-6, 0.0, 0.0, 0.0, 0.0, 0x1.1111111111111p-5, -0x1.4e0b29174ffc1p-3, 0x1.1634feb5b82f0p-5, 0x1.4202d1f0f5b35p-3, 0x1.b8c8cd1850248p-3, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
  0x1.2e342198e9114p-5, 0.0, 0.0, 0.0, 0.0, -0x1.2c11b63bca539p-3, 0x1.cb47a94a6dac5p-3, 0x1.77ea59cbdfec1p-6, -0x1.d5e4d0f53f260p-9, 0x1.6317652422c98p-4, 0x1.c0e7c09c6e85fp-2, 0.0, 0.0, 0.0, 0.0, 0.0,
  -0x1.f247973256de2p-2, 0.0, 0.0, 0.0, 0.0, -0x1.937e9c1d4f589p+2, -0x1.1ffed9f2c94dcp-2, -0x1.56ea1a3275a6bp+1, 0x1.09a234ea69dfap-1, 0x1.5d87c9583ee69p+0, 0x1.78a55517c6c06p+2, 0x1.66c27034fd6f7p+1, 0.0, 0.0, 0.0, 0.0,
  0x1.ac94e58d1e167p-2, 0.0, 0.0, 0.0, 0.0, 0x1.ae5efcd22bc8bp+2, -0x1.b3a7aa564f1f2p-2, 0x1.abf0923fc4fe7p+1, 0x1.3bf220b41a2b7p-1, -0x1.dc2485116b775p-1, -0x1.86658fabeb833p+2, -0x1.80484ad86ab9fp+1, 0x1.0572ac219c10cp-2, 0.0, 0.0, 0.0,
  -0x1.8f0a1ec67ecfap-1, 0.0, 0.0, 0.0, 0.0, -0x1.bdfeb5c74a523p+3, 0x1.4086460e4235ep+0, -0x1.d620c576b34cap+3, -0x1.fa93f67e432e5p-2, 0x1.1f19cd44440d6p+1, 0x1.abc5c939fb0acp+3, 0x1.ccb15c5c836e1p+3, -0x1.985c949bcbe2ep-1, 0x1.c3848fd794123p-2, 0.0, 0.0,
  0x1.076e39e9f4653p+1, 0.0, 0.0, 0.0, 0.0, 0x1.65ba1ce93a093p+4, 0x1.d1a9bc7c3cdb6p-1, 0x1.1f20f98d46d29p+5, -0x1.b8a45519d15a4p+1, -0x1.37640bec04168p+2, -0x1.2e8e8e718f1f2p+4, -0x1.121bbd355f980p+5, 0x1.43c7155a15e35p+0, 0.0, 0.0, 0.0,
};
static const double ref_vern9_b[16] = {0x1.dece255e50a69p-7, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -0x1.90eaee0a3fef2p-2, 0x1.d9476af99b058p-3, 0x1.05127df5b7ad1p-3, 0x1.cc11d91f87e5ap-3, 0x1.2309f29447a78p-1, 0x1.dd4161c2dc3f7p-5, 0x1.1769863774af7p-3, 0x1.f4dc75b3aef35p-6, 0.0};
static const double ref_vern9_e[16] = {-0x1.5f24207ad4dafp-8, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -0x1.4aa06a5b4365ap+1, 0x1.23e2da5f7ecf5p-3, 0x1.b7c499f6c6ea1p-7, -0x1.d5c71f7fb597fp-6, 0x1.4ffffd1b94e09p+1, -0x1.21550a3cfce7cp-2, 0x1.1769863774af7p-3, 0x1.f4dc75b3aef35p-6, -0x1.8c052e109946cp-5};
